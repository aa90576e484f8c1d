/*
 * graph_api.c -- the drop-in graph API (include/graph.h) over the CUDA engine.
 *
 * Host side: the same struct graph, field for field, as the reference
 * (graph.c:12-70 allocates it; this file does too, with calloc so that slots
 * the reference leaves uninitialised read as zero).  Construction and
 * bookkeeping functions behave as the reference's; the differences are that
 * edges are bucketed by a stable counting sort instead of hsearch tables with
 * MAX_DEGREE slots (no per-node cap, same order), and init_levels_to_nodes is
 * O(V+E) (same lists).
 *
 * Propagation: every propagate entry point runs on the GPU through bp.h.  The
 * device copy of the graph is built on first use and rebuilt after any
 * structural change.  In the default eager mode each call uploads the host
 * fields it reads and writes back the ones it changes, so callers that read
 * or write struct graph fields directly (the parsers, the drivers, the
 * reference's example) see exactly the reference's state after every call.
 */
#include <assert.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bp.h"
#include "bp_levels.h"
#include "graph.h"

#define BP_CHECK(cond)                                                                            \
    do {                                                                                          \
        if (!(cond)) {                                                                            \
            fprintf(stderr, "%s:%d: %s: Assertion `%s' failed.\n", __FILE__, __LINE__, __func__, \
                    #cond);                                                                       \
            abort();                                                                              \
        }                                                                                         \
    } while (0)

/* device side of one struct graph */
struct bp_side {
    bp_graph *dev;
    int sync_mode;        /* bp_sync_mode */
    int host_stale;       /* device holds newer beliefs/messages/visited */
    int device_stale;     /* host holds newer state than the device */
    int structure_dirty;  /* edges or state counts changed since the device copy was built */
    int src_csr_ready, dest_csr_ready;
};

static struct bp_side *side_of(Graph_t g)
{
    if (!g->bp_device) {
        g->bp_device = calloc(1, sizeof(struct bp_side));
        BP_CHECK(g->bp_device != NULL);
        ((struct bp_side *)g->bp_device)->device_stale = 1;
        ((struct bp_side *)g->bp_device)->structure_dirty = 1;
    }
    return (struct bp_side *)g->bp_device;
}

static void die_bp(int st, const char *what)
{
    fprintf(stderr, "belief propagation engine: %s failed: %s (%s)\n", what, bp_status_string(st),
            bp_last_error());
    abort();
}

#define BP_CALL(expr)                   \
    do {                                \
        int st_ = (expr);               \
        if (st_ != BP_OK)               \
            die_bp(st_, #expr);         \
    } while (0)

static void mark_structure(Graph_t g)
{
    struct bp_side *s = side_of(g);
    s->structure_dirty = 1;
    s->device_stale = 1;
}

static void sync_host_now(Graph_t g);

/* before a host-side mutation in lazy mode, bring the host up to date */
static void before_host_write(Graph_t g)
{
    struct bp_side *s = side_of(g);
    if (s->host_stale)
        sync_host_now(g);
    s->device_stale = 1;
}

Graph_t create_graph(unsigned int num_vertices, unsigned int num_edges)
{
    Graph_t g = (Graph_t)calloc(1, sizeof(struct graph));
    BP_CHECK(g);
    size_t V = num_vertices ? num_vertices : 1, E = num_edges ? num_edges : 1;
    g->edges_src_index = (unsigned int *)calloc(E, sizeof(unsigned int));
    g->edges_dest_index = (unsigned int *)calloc(E, sizeof(unsigned int));
    g->edges_x_dim = (unsigned int *)calloc(E, sizeof(unsigned int));
    g->edges_y_dim = (unsigned int *)calloc(E, sizeof(unsigned int));
    g->edges_joint_probabilities = (float *)calloc(E * MAX_STATES * MAX_STATES, sizeof(float));
    g->edges_messages = (float *)calloc(E * MAX_STATES, sizeof(float));
    g->last_edges_messages = (float *)calloc(E * MAX_STATES, sizeof(float));
    g->node_states = (float *)calloc(V * MAX_STATES, sizeof(float));
    g->node_num_vars = (unsigned int *)calloc(V, sizeof(unsigned int));
    g->src_nodes_to_edges_node_list = (unsigned int *)calloc(V, sizeof(unsigned int));
    g->src_nodes_to_edges_edge_list = (unsigned int *)calloc(E, sizeof(unsigned int));
    g->dest_nodes_to_edges_node_list = (unsigned int *)calloc(V, sizeof(unsigned int));
    g->dest_nodes_to_edges_edge_list = (unsigned int *)calloc(E, sizeof(unsigned int));
    g->node_names = (char *)calloc(V * CHAR_BUFFER_SIZE, 1);
    g->visited = (char *)calloc(V, 1);
    g->observed_nodes = (char *)calloc(V, 1);
    g->variable_names = (char *)calloc(V * CHAR_BUFFER_SIZE * MAX_STATES, 1);
    g->levels_to_nodes = (unsigned int *)calloc(2 * V, sizeof(unsigned int));
    BP_CHECK(g->edges_src_index && g->edges_dest_index && g->edges_x_dim && g->edges_y_dim);
    BP_CHECK(g->edges_joint_probabilities && g->edges_messages && g->last_edges_messages);
    BP_CHECK(g->node_states && g->node_num_vars && g->node_names && g->visited && g->observed_nodes);
    BP_CHECK(g->src_nodes_to_edges_node_list && g->src_nodes_to_edges_edge_list);
    BP_CHECK(g->dest_nodes_to_edges_node_list && g->dest_nodes_to_edges_edge_list);
    BP_CHECK(g->variable_names && g->levels_to_nodes);

    g->current_edge_messages = &g->edges_messages;
    g->previous_edge_messages = &g->last_edges_messages;
    g->node_hash_table_created = 0;
    g->edge_tables_created = 0;
    g->num_levels = 0;
    g->total_num_vertices = num_vertices;
    g->total_num_edges = num_edges;
    g->current_num_vertices = 0;
    g->current_num_edges = 0;
    g->diameter = -1;
    g->max_degree = 0;
    g->bp_device = NULL;
    return g;
}

void initialize_node(Graph_t graph, unsigned int node_index, unsigned int num_variables)
{
    before_host_write(graph);
    for (unsigned int i = 0; i < num_variables; ++i)
        graph->node_states[node_index * MAX_STATES + i] = DEFAULT_STATE;
    graph->node_num_vars[node_index] = num_variables;
    mark_structure(graph);
}

void init_edge(Graph_t graph, unsigned int edge_index, unsigned int src_index, unsigned int dest_index,
               unsigned int dim_x, unsigned int dim_y, float *joint_probabilities)
{
    BP_CHECK(dim_x <= MAX_STATES);
    BP_CHECK(dim_y <= MAX_STATES);
    before_host_write(graph);
    graph->edges_src_index[edge_index] = src_index;
    graph->edges_dest_index[edge_index] = dest_index;
    graph->edges_x_dim[edge_index] = dim_x;
    graph->edges_y_dim[edge_index] = dim_y;
    for (unsigned int i = 0; i < dim_x; ++i) {
        for (unsigned int j = 0; j < dim_y; ++j)
            graph->edges_joint_probabilities[(size_t)MAX_STATES * MAX_STATES * edge_index + MAX_STATES * i + j] =
                joint_probabilities[MAX_STATES * i + j];
        graph->edges_messages[(size_t)MAX_STATES * edge_index + i] = 0;
        graph->last_edges_messages[(size_t)MAX_STATES * edge_index + i] = 0;
    }
    mark_structure(graph);
}

void node_set_state(Graph_t graph, unsigned int node_index, unsigned int num_variables, float *state)
{
    before_host_write(graph);
    for (unsigned int i = 0; i < num_variables; ++i)
        graph->node_states[node_index * MAX_STATES + i] = state[i];
}

void graph_add_node(Graph_t g, unsigned int num_variables, const char *name)
{
    unsigned int node_index = g->current_num_vertices;
    BP_CHECK(node_index < g->total_num_vertices);
    initialize_node(g, node_index, num_variables);
    strncpy(&g->node_names[node_index * CHAR_BUFFER_SIZE], name, CHAR_BUFFER_SIZE);
    g->current_num_vertices += 1;
}

void graph_add_and_set_node_state(Graph_t g, unsigned int num_variables, const char *name, float *state)
{
    unsigned int node_index = g->current_num_vertices;
    g->observed_nodes[node_index] = 1;
    graph_add_node(g, num_variables, name);
    node_set_state(g, node_index, num_variables, state);
}

void graph_set_node_state(Graph_t g, unsigned int node_index, unsigned int num_states, float *state)
{
    BP_CHECK(node_index < g->current_num_vertices);
    BP_CHECK(num_states <= g->node_num_vars[node_index]);
    g->observed_nodes[node_index] = 1;
    node_set_state(g, node_index, num_states, state);
}

void graph_add_edge(Graph_t graph, unsigned int src_index, unsigned int dest_index, unsigned int dim_x,
                    unsigned int dim_y, float *joint_probabilities)
{
    unsigned int edge_index = graph->current_num_edges;
    BP_CHECK(edge_index < graph->total_num_edges);
    BP_CHECK(graph->node_num_vars[src_index] == dim_x);
    BP_CHECK(graph->node_num_vars[dest_index] == dim_y);
    init_edge(graph, edge_index, src_index, dest_index, dim_x, dim_y, joint_probabilities);
    graph->edge_tables_created = 1;
    graph->current_num_edges += 1;
}

void fill_in_node_hash_table(Graph_t graph)
{
    ENTRY e, *ep;
    if (graph->node_hash_table_created == 0) {
        graph->node_hash_table = (struct hsearch_data *)calloc(sizeof(struct hsearch_data), 1);
        BP_CHECK(graph->node_hash_table);
        hcreate_r(graph->current_num_vertices, graph->node_hash_table);
        for (unsigned int i = 0; i < graph->current_num_vertices; ++i) {
            e.key = &(graph->node_names[i * CHAR_BUFFER_SIZE]);
            e.data = (void *)(uintptr_t)i;
            BP_CHECK(hsearch_r(e, ENTER, &ep, graph->node_hash_table) != 0);
        }
        graph->node_hash_table_created = 1;
    }
}

void fill_in_node_table(Graph_t graph) { fill_in_node_hash_table(graph); }

unsigned int find_node_by_name(char *name, Graph_t graph)
{
    ENTRY e, *ep;
    fill_in_node_hash_table(graph);
    e.key = name;
    BP_CHECK(hsearch_r(e, FIND, &ep, graph->node_hash_table) != 0);
    BP_CHECK(ep != NULL);
    unsigned int i = (unsigned int)(uintptr_t)ep->data;
    BP_CHECK(i < graph->current_num_vertices);
    return i;
}

/* stable counting sort of the current edges by key into node_list (V row
 * starts, the reference's layout: the last row ends at current_num_edges) and
 * edge_list; returns the largest row length */
static unsigned int bucket_edges(Graph_t g, const unsigned int *key, unsigned int *node_list, unsigned int *edge_list)
{
    unsigned int V = g->current_num_vertices, E = g->current_num_edges, max_deg = 0;
    unsigned int *cnt = (unsigned int *)calloc((size_t)V + 1, sizeof(unsigned int));
    BP_CHECK(cnt);
    for (unsigned int e = 0; e < E; ++e) {
        BP_CHECK(key[e] < V);
        cnt[key[e] + 1]++;
    }
    for (unsigned int v = 0; v < V; ++v) {
        if (cnt[v + 1] > max_deg)
            max_deg = cnt[v + 1];
        cnt[v + 1] += cnt[v];
    }
    for (unsigned int v = 0; v < V; ++v)
        node_list[v] = cnt[v];
    for (unsigned int e = 0; e < E; ++e)
        edge_list[cnt[key[e]]++] = e;
    free(cnt);
    return max_deg;
}

/* graph.c:249-283 */
void set_up_src_nodes_to_edges(Graph_t graph)
{
    BP_CHECK(graph->current_num_vertices == graph->total_num_vertices);
    BP_CHECK(graph->current_num_edges <= graph->total_num_edges);
    unsigned int md = bucket_edges(graph, graph->edges_src_index, graph->src_nodes_to_edges_node_list,
                                   graph->src_nodes_to_edges_edge_list);
    if (md > graph->max_degree)
        graph->max_degree = md;
    side_of(graph)->src_csr_ready = 1;
    mark_structure(graph);
}

/* graph.c:285-313 */
void set_up_dest_nodes_to_edges(Graph_t graph)
{
    BP_CHECK(graph->current_num_vertices == graph->total_num_vertices);
    BP_CHECK(graph->current_num_edges <= graph->total_num_edges);
    bucket_edges(graph, graph->edges_dest_index, graph->dest_nodes_to_edges_node_list,
                 graph->dest_nodes_to_edges_edge_list);
    side_of(graph)->dest_csr_ready = 1;
    mark_structure(graph);
}

int graph_vertex_count(Graph_t g) { return g->current_num_vertices; }

int graph_edge_count(Graph_t g) { return g->current_num_edges; }

void graph_destroy(Graph_t g)
{
    if (g->node_hash_table_created != 0) {
        hdestroy_r(g->node_hash_table);
        free(g->node_hash_table);
    }
    if (g->bp_device) {
        struct bp_side *s = (struct bp_side *)g->bp_device;
        if (s->dev)
            bp_graph_destroy(s->dev);
        free(s);
    }
    free(g->edges_src_index);
    free(g->edges_dest_index);
    free(g->edges_x_dim);
    free(g->edges_y_dim);
    free(g->edges_joint_probabilities);
    free(g->edges_messages);
    free(g->last_edges_messages);
    free(g->src_nodes_to_edges_node_list);
    free(g->src_nodes_to_edges_edge_list);
    free(g->dest_nodes_to_edges_node_list);
    free(g->dest_nodes_to_edges_edge_list);
    free(g->node_names);
    free(g->visited);
    free(g->observed_nodes);
    free(g->variable_names);
    free(g->levels_to_nodes);
    free(g->node_num_vars);
    free(g->node_states);
    free(g);
}

/* ------------------------------------------------------------------ device */

static bp_graph *device_graph(Graph_t g)
{
    struct bp_side *s = side_of(g);
    if (s->dev && !s->structure_dirty)
        return s->dev;
    if (s->dev) {
        bp_graph_destroy(s->dev);
        s->dev = NULL;
    }
    bp_graph_desc d;
    memset(&d, 0, sizeof d);
    d.num_nodes = g->current_num_vertices;
    d.num_edges = g->current_num_edges;
    d.node_num_states = g->node_num_vars;
    d.edge_src = g->edges_src_index;
    d.edge_dst = g->edges_dest_index;
    d.edge_joint = g->edges_joint_probabilities;
    d.joint_row_stride = MAX_STATES;
    d.joint_edge_stride = MAX_STATES * MAX_STATES;
    if (s->dest_csr_ready) {
        d.dest_node_list = g->dest_nodes_to_edges_node_list;
        d.dest_edge_list = g->dest_nodes_to_edges_edge_list;
    }
    d.memory = BP_MEM_HOST;
    BP_CALL(bp_graph_create(&s->dev, &d, NULL));
    s->structure_dirty = 0;
    s->device_stale = 1;
    return s->dev;
}

static int latest_slot(Graph_t g) { return *g->previous_edge_messages == g->edges_messages ? 0 : 1; }

static void set_latest_slot(Graph_t g, int slot)
{
    if (slot == 0) {
        g->previous_edge_messages = &g->edges_messages;
        g->current_edge_messages = &g->last_edges_messages;
    } else {
        g->previous_edge_messages = &g->last_edges_messages;
        g->current_edge_messages = &g->edges_messages;
    }
}

enum { SYNC_BELIEFS = 1, SYNC_MSG0 = 2, SYNC_MSG1 = 4, SYNC_VISITED = 8, SYNC_ALL = 15 };

static void upload(Graph_t g, int what)
{
    struct bp_side *s = side_of(g);
    bp_graph *d = device_graph(g);
    if (s->sync_mode == BP_SYNC_LAZY && !s->device_stale)
        return;
    if (s->sync_mode == BP_SYNC_LAZY)
        what = SYNC_ALL;
    if (what & SYNC_BELIEFS)
        BP_CALL(bp_set_beliefs(d, g->node_states, MAX_STATES, BP_MEM_HOST));
    if (what & SYNC_MSG0)
        BP_CALL(bp_set_messages(d, 0, g->edges_messages, MAX_STATES, BP_MEM_HOST));
    if (what & SYNC_MSG1)
        BP_CALL(bp_set_messages(d, 1, g->last_edges_messages, MAX_STATES, BP_MEM_HOST));
    if (what & SYNC_VISITED)
        BP_CALL(bp_set_visited(d, g->visited));
    BP_CALL(bp_set_latest_slot(d, latest_slot(g)));
    s->device_stale = 0;
}

static void download(Graph_t g, int what, int force)
{
    struct bp_side *s = side_of(g);
    bp_graph *d = s->dev;
    int slot = 0;
    if (!d)
        return;
    if (s->sync_mode == BP_SYNC_LAZY && !force) {
        s->host_stale = 1;
        return;
    }
    if (what & SYNC_BELIEFS)
        BP_CALL(bp_get_beliefs(d, g->node_states, MAX_STATES, BP_MEM_HOST));
    if (what & SYNC_MSG0)
        BP_CALL(bp_get_messages(d, 0, g->edges_messages, MAX_STATES, BP_MEM_HOST));
    if (what & SYNC_MSG1)
        BP_CALL(bp_get_messages(d, 1, g->last_edges_messages, MAX_STATES, BP_MEM_HOST));
    if (what & SYNC_VISITED)
        BP_CALL(bp_get_visited(d, g->visited));
    BP_CALL(bp_get_latest_slot(d, &slot));
    set_latest_slot(g, slot);
    if (what == SYNC_ALL)
        s->host_stale = 0;
}

static void sync_host_now(Graph_t g)
{
    struct bp_side *s = side_of(g);
    if (s->dev && s->host_stale) {
        int mode = s->sync_mode;
        s->sync_mode = BP_SYNC_EAGER;
        download(g, SYNC_ALL, 1);
        s->sync_mode = mode;
    }
    s->host_stale = 0;
}

int bp_set_sync_mode(struct graph *g, int mode)
{
    if (!g || (mode != BP_SYNC_EAGER && mode != BP_SYNC_LAZY))
        return BP_ERR_INVALID;
    struct bp_side *s = side_of(g);
    if (mode == BP_SYNC_EAGER)
        sync_host_now(g);
    s->sync_mode = mode;
    return BP_OK;
}

int bp_sync_host(struct graph *g)
{
    if (!g)
        return BP_ERR_INVALID;
    sync_host_now(g);
    return BP_OK;
}

int bp_graph_of(struct graph *g, bp_graph **out)
{
    if (!g || !out)
        return BP_ERR_INVALID;
    *out = device_graph(g);
    return BP_OK;
}

/* ------------------------------------------------------------- loopy BP */

/* init_previous_edge, graph.c:725-751 */
void init_previous_edge(Graph_t graph)
{
    upload(graph, SYNC_BELIEFS);
    bp_graph *d = device_graph(graph);
    BP_CALL(bp_init_messages(d));
    download(graph, latest_slot(graph) == 0 ? SYNC_MSG0 : SYNC_MSG1, 0);
}

static unsigned int run_loopy(Graph_t graph, float convergence, unsigned int max_iterations, int schedule,
                              unsigned int check_every, int verbose)
{
    upload(graph, SYNC_BELIEFS | SYNC_MSG0 | SYNC_MSG1);
    bp_graph *d = device_graph(graph);
    bp_loopy_options o;
    bp_loopy_default_options(&o);
    o.tolerance = convergence;
    o.max_iterations = max_iterations;
    o.check_every = check_every;
    o.schedule = schedule;
    o.verbose = verbose;
    const char *mode = getenv("BP_DELTA_MODE");
    if (mode && strcmp(mode, "f64") == 0)
        o.delta_mode = BP_DELTA_F64;
    else if (mode && strcmp(mode, "serial") == 0)
        o.delta_mode = BP_DELTA_SERIAL_F32;
    bp_loopy_result r;
    BP_CALL(bp_loopy(d, &o, &r));
    fflush(stdout);
    download(graph, SYNC_BELIEFS | SYNC_MSG0 | SYNC_MSG1, 1);
    return r.iterations;
}

/* loopy_propagate_one_iteration, graph.c:1121-1183 */
void loopy_propagate_one_iteration(Graph_t graph) { run_loopy(graph, -1.0f, 1, BP_SCHEDULE_NODE, 1, 0); }

/* loopy_propagate_until, graph.c:1278-1324 */
unsigned int loopy_propagate_until(Graph_t graph, float convergence, unsigned int max_iterations)
{
    return run_loopy(graph, convergence, max_iterations, BP_SCHEDULE_NODE, 1, 1);
}

/* loopy_propagate_until_edge, graph.c:1230-1276 */
unsigned int loopy_propagate_until_edge(Graph_t graph, float convergence, unsigned int max_iterations)
{
    return run_loopy(graph, convergence, max_iterations, BP_SCHEDULE_EDGE, 1, 1);
}

/* loopy_progagate_until_acc (sic), graph.c:1422-1442 */
unsigned int loopy_progagate_until_acc(Graph_t graph, float convergence, unsigned int max_iterations)
{
    return run_loopy(graph, convergence, max_iterations, BP_SCHEDULE_NODE, BATCH_SIZE, 1);
}

/* loopy_progagate_until_edge_acc (sic), graph.c:1527-1547 */
unsigned int loopy_progagate_until_edge_acc(Graph_t graph, float convergence, unsigned int max_iterations)
{
    return run_loopy(graph, convergence, max_iterations, BP_SCHEDULE_EDGE, BATCH_SIZE, 1);
}

/* -------------------------------------------------------------- tree BP */

static void tree_levels_to_device(Graph_t g)
{
    bp_graph *d = device_graph(g);
    BP_CALL(bp_tree_set_levels(d, g->levels_to_nodes, g->num_levels));
}

/* graph.c:376-424 */
void propagate_using_levels_start(Graph_t g)
{
    upload(g, SYNC_BELIEFS | SYNC_MSG0 | SYNC_VISITED);
    tree_levels_to_device(g);
    BP_CALL(bp_tree_start(device_graph(g)));
    download(g, SYNC_MSG0 | SYNC_VISITED, 0);
}

/* graph.c:524-538 */
void propagate_using_levels(Graph_t g, unsigned int current_level)
{
    upload(g, SYNC_MSG0 | SYNC_VISITED);
    tree_levels_to_device(g);
    BP_CALL(bp_tree_level(device_graph(g), current_level));
    download(g, SYNC_MSG0 | SYNC_VISITED, 0);
}

/* graph.c:588-596 */
void marginalize(Graph_t g)
{
    upload(g, SYNC_BELIEFS | SYNC_MSG0);
    BP_CALL(bp_tree_marginalize(device_graph(g)));
    download(g, SYNC_ALL, 1);
}

/* graph.c:598-605 */
void reset_visited(Graph_t g)
{
    struct bp_side *s = side_of(g);
    if (s->sync_mode == BP_SYNC_LAZY && s->dev && !s->device_stale) {
        BP_CALL(bp_tree_reset_visited(s->dev));
        if (s->host_stale) {
            memset(g->visited, 0, g->current_num_vertices);
            return;
        }
    }
    for (unsigned int i = 0; i < g->current_num_vertices; ++i)
        g->visited[i] = 0;
}

/* graph.c:753-772 */
void fill_in_leaf_nodes_in_index(Graph_t graph, unsigned int *start_index, unsigned int *end_index,
                                 unsigned int max_count)
{
    graph->levels_to_nodes[0] = *start_index;
    for (unsigned int i = 0; i < graph->current_num_vertices; ++i) {
        unsigned int lo = graph->dest_nodes_to_edges_node_list[i];
        unsigned int hi = (i + 1 == graph->current_num_vertices) ? graph->current_num_edges
                                                                  : graph->dest_nodes_to_edges_node_list[i + 1];
        if (hi - lo <= max_count) {
            graph->levels_to_nodes[*end_index] = i;
            *end_index += 1;
        }
    }
}

/* graph.c:774-804 (same appends; the duplicate check scans the list as the
 * reference does -- this entry point is kept for callers that drive it
 * themselves; init_levels_to_nodes below uses the O(V+E) form) */
void visit_node(Graph_t graph, unsigned int buffer_index, unsigned int *end_index)
{
    unsigned int node_index = graph->levels_to_nodes[buffer_index];
    if (graph->visited[node_index] != 0)
        return;
    graph->visited[node_index] = 1;
    unsigned int lo = graph->src_nodes_to_edges_node_list[node_index];
    unsigned int hi = (node_index + 1 == graph->current_num_vertices) ? graph->current_num_edges
                                                                       : graph->src_nodes_to_edges_node_list[node_index + 1];
    for (unsigned int i = lo; i < hi; ++i) {
        unsigned int dest = graph->edges_dest_index[graph->src_nodes_to_edges_edge_list[i]];
        int listed = 0;
        for (unsigned int j = graph->current_num_vertices; j < *end_index; ++j)
            if (graph->levels_to_nodes[j] == dest) {
                listed = 1;
                break;
            }
        if (!listed) {
            graph->levels_to_nodes[*end_index] = dest;
            *end_index += 1;
        }
    }
}

/* graph.c:806-827, in O(V+E) */
void init_levels_to_nodes(Graph_t graph)
{
    unsigned int V = graph->current_num_vertices, E = graph->current_num_edges;
    reset_visited(graph);
    unsigned int *in_ptr = (unsigned int *)malloc(sizeof(unsigned int) * ((size_t)V + 1));
    unsigned int *out_ptr = (unsigned int *)malloc(sizeof(unsigned int) * ((size_t)V + 1));
    unsigned int *out_dst = (unsigned int *)malloc(sizeof(unsigned int) * (E ? E : 1));
    BP_CHECK(in_ptr && out_ptr && out_dst);
    for (unsigned int v = 0; v < V; ++v) {
        in_ptr[v] = graph->dest_nodes_to_edges_node_list[v];
        out_ptr[v] = graph->src_nodes_to_edges_node_list[v];
    }
    in_ptr[V] = E;
    out_ptr[V] = E;
    for (unsigned int q = 0; q < E; ++q)
        out_dst[q] = graph->edges_dest_index[graph->src_nodes_to_edges_edge_list[q]];
    int rc = bp_levels_from_csr(V, in_ptr, out_ptr, out_dst, graph->levels_to_nodes, &graph->num_levels);
    free(in_ptr);
    free(out_ptr);
    free(out_dst);
    if (rc == -1) {
        fprintf(stderr, "init_levels_to_nodes: some nodes are unreachable from the nodes with in-degree <= 2 "
                        "(the reference loops forever here)\n");
        abort();
    }
    BP_CHECK(rc == 0);
    reset_visited(graph);
}

/* ------------------------------------------------------------- printing */

static void ensure_host(Graph_t g)
{
    if (g->bp_device && ((struct bp_side *)g->bp_device)->host_stale)
        sync_host_now(g);
}

void print_node(Graph_t graph, unsigned int node_index)
{
    ensure_host(graph);
    unsigned int num_vars = graph->node_num_vars[node_index];
    printf("Node %s [\n", &graph->node_names[node_index * CHAR_BUFFER_SIZE]);
    for (unsigned int i = 0; i < num_vars; ++i) {
        unsigned int k = node_index * CHAR_BUFFER_SIZE * MAX_STATES + i * CHAR_BUFFER_SIZE;
        printf("%s:\t%.6lf\n", &graph->variable_names[k], graph->node_states[MAX_STATES * node_index + i]);
    }
    printf("]\n");
}

void print_edge(Graph_t graph, unsigned int edge_index)
{
    ensure_host(graph);
    unsigned int dim_x = graph->edges_x_dim[edge_index], dim_y = graph->edges_y_dim[edge_index];
    unsigned int src_index = graph->edges_src_index[edge_index], dest_index = graph->edges_dest_index[edge_index];
    printf("Edge  %s -> %s [\n", &graph->node_names[src_index * CHAR_BUFFER_SIZE],
           &graph->node_names[dest_index * CHAR_BUFFER_SIZE]);
    printf("Joint probability matrix: [\n");
    for (unsigned int i = 0; i < dim_x; ++i) {
        printf("[");
        for (unsigned int j = 0; j < dim_y; ++j)
            printf("\t%.6lf",
                   graph->edges_joint_probabilities[(size_t)MAX_STATES * MAX_STATES * edge_index + MAX_STATES * i + j]);
        printf("\t]\n");
    }
    printf("]\nMessage:\n[");
    for (unsigned int i = 0; i < dim_x; ++i)
        printf("\t%.6lf", graph->edges_messages[(size_t)MAX_STATES * edge_index + i]);
    printf("\t]\n]\n");
}

void print_nodes(Graph_t g)
{
    for (unsigned int i = 0; i < g->current_num_vertices; ++i)
        print_node(g, i);
}

void print_edges(Graph_t g)
{
    for (unsigned int i = 0; i < g->current_num_edges; ++i)
        print_edge(g, i);
}

static void print_csr(Graph_t g, const unsigned int *nodes, const unsigned int *edges)
{
    unsigned int V = g->total_num_vertices;
    for (unsigned int i = 0; i < V; ++i) {
        printf("Node -----\n");
        print_node(g, i);
        printf("Edges-------\n");
        unsigned int lo = nodes[i], hi = (i + 1 == V) ? g->current_num_edges : nodes[i + 1];
        for (unsigned int j = lo; j < hi; ++j)
            print_edge(g, edges[j]);
        printf("---------\n");
    }
}

void print_src_nodes_to_edges(Graph_t g)
{
    printf("src index -> edge index\n");
    print_csr(g, g->src_nodes_to_edges_node_list, g->src_nodes_to_edges_edge_list);
}

void print_dest_nodes_to_edges(Graph_t g)
{
    printf("dest index -> edge index\n");
    print_csr(g, g->dest_nodes_to_edges_node_list, g->dest_nodes_to_edges_edge_list);
}

void print_levels_to_nodes(Graph_t graph)
{
    for (unsigned int i = 0; i < graph->num_levels; ++i) {
        printf("Level: %d\n", i);
        printf("---------------\n");
        unsigned int lo = graph->levels_to_nodes[i];
        unsigned int hi = (i + 1 == graph->num_levels) ? graph->current_num_vertices * 2 : graph->levels_to_nodes[i + 1];
        printf("Nodes:-----------\n");
        for (unsigned int j = lo; j < hi; ++j)
            print_node(graph, graph->levels_to_nodes[j]);
        printf("-------------------\n");
    }
}

/* send_message (graph.c:426-448) is exported by the reference; kept as the
 * same host function for callers that use it directly */
void send_message(float *states, unsigned int offset, unsigned int edge_index, float *edge_joint_probabilities,
                  float *edge_messages, unsigned int *edge_num_src, unsigned int *edge_num_dest)
{
    unsigned int num_src = edge_num_src[edge_index], num_dest = edge_num_dest[edge_index];
    float sum = 0.0f;
    for (unsigned int i = 0; i < num_src; ++i) {
        float partial = 0.0f;
        for (unsigned int j = 0; j < num_dest; ++j)
            partial += edge_joint_probabilities[(size_t)MAX_STATES * MAX_STATES * edge_index + MAX_STATES * i + j] *
                       states[offset + j];
        edge_messages[(size_t)MAX_STATES * edge_index + i] = partial;
        sum += partial;
    }
    if (sum <= 0.0f)
        sum = 1.0f;
    for (unsigned int i = 0; i < num_src; ++i)
        edge_messages[(size_t)MAX_STATES * edge_index + i] = edge_messages[(size_t)MAX_STATES * edge_index + i] / sum;
}

/* calculate_diameter, graph.c:1549-1618: the largest finite shortest-path
 * length over ordered pairs (i, j), paths of at least one edge, so a node's
 * shortest cycle counts for (i, i).  The reference runs Floyd-Warshall on
 * V x V matrices; one BFS per source gives the same number in O(V (V + E)). */
void calculate_diameter(Graph_t graph)
{
    unsigned int V = graph->current_num_vertices, E = graph->current_num_edges;
    int *dist = (int *)malloc(sizeof(int) * (V ? V : 1));
    unsigned int *queue = (unsigned int *)malloc(sizeof(unsigned int) * (V ? V : 1));
    BP_CHECK(dist && queue);
    graph->diameter = -1;
    for (unsigned int s = 0; s < V; ++s) {
        for (unsigned int v = 0; v < V; ++v)
            dist[v] = -1;
        unsigned int head = 0, tail = 0;
        /* seed with the out-neighbours of s at distance 1; s itself is not
         * at distance 0 (the reference's matrix has no zero diagonal) */
        unsigned int lo = graph->src_nodes_to_edges_node_list[s];
        unsigned int hi = (s + 1 == V) ? E : graph->src_nodes_to_edges_node_list[s + 1];
        for (unsigned int q = lo; q < hi; ++q) {
            unsigned int w = graph->edges_dest_index[graph->src_nodes_to_edges_edge_list[q]];
            if (dist[w] < 0) {
                dist[w] = 1;
                queue[tail++] = w;
            }
        }
        while (head < tail) {
            unsigned int u = queue[head++];
            unsigned int a = graph->src_nodes_to_edges_node_list[u];
            unsigned int b = (u + 1 == V) ? E : graph->src_nodes_to_edges_node_list[u + 1];
            for (unsigned int q = a; q < b; ++q) {
                unsigned int w = graph->edges_dest_index[graph->src_nodes_to_edges_edge_list[q]];
                if (dist[w] < 0) {
                    dist[w] = dist[u] + 1;
                    queue[tail++] = w;
                }
            }
        }
        for (unsigned int v = 0; v < V; ++v)
            if (dist[v] >= 0 && dist[v] < WEIGHT_INFINITY && dist[v] > graph->diameter)
                graph->diameter = dist[v];
    }
    free(dist);
    free(queue);
}
