/*
 * graph.h -- drop-in replacement for the reference's C graph API
 * (src/graph/graph.h:20-133), backed by sm_100a CUDA kernels.
 *
 * ABI contract
 * ------------
 * Callers read and write the fields of struct graph directly (the BIF parser
 * expression.c:245-248,636-640,706-762,906-913; the XMLBIF parser
 * xml-expression.c:152-161,361-409; the benchmark drivers c_benchmark/main.c;
 * example-belief-propagation.c:30-105).  Every field therefore keeps the
 * reference's name, type, order and host layout:
 *   node_states            [V][MAX_STATES] beliefs (host, valid after every
 *                          propagate call)
 *   edges_joint_probabilities [E][MAX_STATES][MAX_STATES]
 *   edges_messages / last_edges_messages [E][MAX_STATES], with
 *                          *previous_edge_messages pointing at the latest
 *                          messages after a loopy iteration (graph.c:1180-1182)
 *   levels_to_nodes        [2V]: level offsets in [0, num_levels), node ids
 *                          in [V, 2V) (graph.c:806-827)
 * One field is appended at the end: `bp_device`, an opaque pointer to the
 * device-resident copy of the graph.  Callers never allocate struct graph
 * themselves (create_graph does), so code compiled against the reference's
 * header links against this library unchanged.
 *
 * Host/device synchronisation: by default every propagate entry point uploads
 * the host fields it reads and writes back the ones it changes, so direct
 * field access keeps working.  bp_set_sync_mode() in bp.h switches a graph to
 * lazy mode, where the device copy stays authoritative between calls and the
 * host fields are refreshed by loopy_propagate_*, marginalize, the print_*
 * functions and bp_sync_host().
 *
 * Behaviour differences from the reference:
 *  - no MAX_DEGREE cap on per-node edge lists;
 *  - graphs whose nodes have different state counts use zero padding where
 *    the reference reads uninitialised buffer slots (graph.c:462,481-483,
 *    851-857);
 *  - init_levels_to_nodes is O(V+E) instead of O(V^2) and produces the same
 *    level lists.
 */

#ifndef GRAPH_H_
#define GRAPH_H_

#ifndef __USE_GNU
#define __USE_GNU
#endif

#include "constants.h"

#include <search.h>

#ifdef __cplusplus
extern "C" {
#endif

struct graph {
	unsigned int total_num_vertices;
	unsigned int total_num_edges;

	unsigned int current_num_vertices;
	unsigned int current_num_edges;
	unsigned int max_degree;

	unsigned int * edges_src_index;
	unsigned int * edges_dest_index;
	unsigned int * edges_x_dim;
	unsigned int * edges_y_dim;
	float * edges_joint_probabilities;

	float * edges_messages;
	float * last_edges_messages;

	float ** current_edge_messages;
	float ** previous_edge_messages;

	float * node_states;
	unsigned int * node_num_vars;

	unsigned int * src_nodes_to_edges_node_list;
	unsigned int * src_nodes_to_edges_edge_list;

	unsigned int * dest_nodes_to_edges_node_list;
	unsigned int * dest_nodes_to_edges_edge_list;

	unsigned int * levels_to_nodes;
	unsigned int num_levels;

	int diameter;

	char * visited;
	char * node_names;

	char * variable_names;

	char * observed_nodes;

	char graph_name[CHAR_BUFFER_SIZE];

	char node_hash_table_created;
	struct hsearch_data *node_hash_table;

	struct hsearch_data *src_node_to_edge_table;

	struct hsearch_data *dest_node_to_edge_table;
	char edge_tables_created;

	/* appended: device-resident mirror owned by this library (opaque) */
	void * bp_device;
};
typedef struct graph* Graph_t;

/* Kept for source compatibility (graph.h:76-79); unused by this library. */
struct htable_entry {
	unsigned int indices[MAX_DEGREE];
	unsigned int count;
};

/* construction -- graph.c:12-313 */
Graph_t create_graph(unsigned int, unsigned int);

void graph_add_node(Graph_t, unsigned int, const char *);
void graph_add_and_set_node_state(Graph_t, unsigned int, const char *, float *);
void graph_set_node_state(Graph_t, unsigned int, unsigned int, float *);

void graph_add_edge(Graph_t, unsigned int, unsigned int, unsigned int, unsigned int, float *);

void set_up_src_nodes_to_edges(Graph_t);
void set_up_dest_nodes_to_edges(Graph_t);
void init_levels_to_nodes(Graph_t);
void calculate_diameter(Graph_t);

void initialize_node(Graph_t, unsigned int, unsigned int);
void node_set_state(Graph_t, unsigned int, unsigned int, float *);

void init_edge(Graph_t, unsigned int, unsigned int, unsigned int, unsigned int, unsigned int, float *);
void send_message(float *, unsigned int, unsigned int, float *, float *, unsigned int *, unsigned int *);

void fill_in_node_table(Graph_t);
unsigned int find_node_by_name(char *, Graph_t);

/* non-static in the reference and called by its parsers / drivers
 * (expression.c:630, graph.c:753, graph.c:774) */
void fill_in_node_hash_table(Graph_t);
void fill_in_leaf_nodes_in_index(Graph_t, unsigned int *, unsigned int *, unsigned int);
void visit_node(Graph_t, unsigned int, unsigned int *);

int graph_vertex_count(Graph_t);
int graph_edge_count(Graph_t);

void graph_destroy(Graph_t);

/* tree BP -- graph.c:376-605 (GPU level-synchronous frontier passes) */
void propagate_using_levels_start(Graph_t);
void propagate_using_levels(Graph_t, unsigned int);

void reset_visited(Graph_t);

/* loopy BP -- graph.c:725-751, :1121-1547 (GPU flooding kernels) */
void init_previous_edge(Graph_t);
void loopy_propagate_one_iteration(Graph_t);

unsigned int loopy_propagate_until(Graph_t, float convergence, unsigned int max_iterations);
unsigned int loopy_propagate_until_edge(Graph_t, float, unsigned int);
unsigned int loopy_progagate_until_acc(Graph_t, float convergence, unsigned int max_iterations);
unsigned int loopy_progagate_until_edge_acc(Graph_t, float, unsigned int);

void marginalize(Graph_t);

void print_node(Graph_t, unsigned int);
void print_edge(Graph_t, unsigned int);
void print_nodes(Graph_t);
void print_edges(Graph_t);
void print_src_nodes_to_edges(Graph_t);
void print_dest_nodes_to_edges(Graph_t);
void print_levels_to_nodes(Graph_t);

#ifdef __cplusplus
}
#endif

#endif /* GRAPH_H_ */
