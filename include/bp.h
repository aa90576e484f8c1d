/*
 * bp.h -- device-resident C-ABI of the B200 belief-propagation engine.
 *
 * graph.h is the drop-in (the reference's API, host struct layout kept);
 * this header is the layer underneath it, usable directly by callers that
 * want the graph to stay in GPU memory between calls, pass device pointers,
 * or run the batched / differentiable modes.  Plain C types only: pointers,
 * sizes, status codes.  `memory` arguments say whether a pointer is host
 * (BP_MEM_HOST) or device (BP_MEM_DEVICE) memory; `stream` arguments are
 * cudaStream_t values passed as void* (NULL = the graph's own stream).
 *
 * Layouts
 *   beliefs   [V][ld]  node v uses slots [0, S_v); slots at or beyond S_v
 *             are read as zero and written as zero
 *   messages  [E][ld]  in edge-id (insertion) order, edge e uses [0, S_src(e))
 *   joint     per edge, rows i < S_src, columns j < S_dst, row stride and
 *             edge stride given by the caller (MAX_STATES and MAX_STATES^2
 *             for struct graph's edges_joint_probabilities)
 *
 * Every entry point returns a bp_status; bp_last_error() gives the message
 * of the most recent failure on the calling thread.
 */
#ifndef BP_H_
#define BP_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BP_MAX_STATES 10

typedef enum {
    BP_OK = 0,
    BP_ERR_INVALID = 1,     /* null pointer, bad enum, index out of range */
    BP_ERR_SHAPE = 2,       /* state count 0 or > BP_MAX_STATES, sizes too large */
    BP_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    BP_ERR_NOMEM = 4,       /* device allocation failed */
    BP_ERR_NO_DEVICE = 5,   /* no CUDA device */
    BP_ERR_GRAPH = 6,       /* tree levels: a node is unreachable from the seed set */
    BP_ERR_STATE = 7,       /* call out of order (e.g. a tree level before levels exist) */
    BP_ERR_TIMEOUT = 8      /* a bounded device wait gave up */
} bp_status;

typedef enum { BP_MEM_HOST = 0, BP_MEM_DEVICE = 1 } bp_memory;

typedef enum {
    BP_SCHEDULE_NODE = 0,   /* loopy_propagate_until / _acc (graph.c:1121, :1326) */
    BP_SCHEDULE_EDGE = 1    /* loopy_propagate_until_edge / _edge_acc (graph.c:1186, :1444) */
} bp_schedule;

typedef enum {
    BP_DELTA_AUTO = 0,       /* SERIAL_F32 up to 2^20 message entries, F64 above */
    BP_DELTA_SERIAL_F32 = 1, /* the reference's own fp32 sum in edge order: same
                                iteration count as the reference, always */
    BP_DELTA_F64 = 2         /* parallel fp64 sum, deterministic order */
} bp_delta_mode;

typedef enum { BP_SYNC_EAGER = 0, BP_SYNC_LAZY = 1 } bp_sync_mode;

/* the node-schedule iteration kernel: same results, different tiling */
typedef enum {
    BP_KERNEL_AUTO = 0,        /* the split schedule for uniform graphs of <= 4 states whose send buffers exceed
                                  64 MB (they no longer stay in L2), else block tiles.  BP_FLOOD_SPLIT=0|1 in the
                                  environment: never | whenever it applies; BP_FLOOD_KERNEL=warp|staged selects warp
                                  tiles, or staged tiles where they apply */
    BP_KERNEL_BLOCK_TILE = 1,  /* 256-node block tiles, block-wide barriers between phases */
    BP_KERNEL_WARP_TILE = 2,   /* 32-node warp tiles, unrolled edge loads */
    BP_KERNEL_STAGED_TILE = 3, /* persistent CTAs, bulk-copy staged tiles; uniform 2-state graphs of mean in-degree
                                  <= 4.5, f64 delta */
    BP_KERNEL_SPLIT = 4        /* send pass over the edges grouped by source-node range (gathers from one
                                  L2-sized range of send buffers at a time) + node pass; uniform graphs of
                                  <= 4 states */
} bp_kernel_variant;

typedef struct bp_graph bp_graph;

typedef struct {
    uint32_t num_nodes;
    uint32_t num_edges;
    uint32_t uniform_states;          /* states of every node when node_num_states is NULL */
    const uint32_t *node_num_states;  /* [num_nodes] or NULL */
    const uint32_t *edge_src;         /* [num_edges] */
    const uint32_t *edge_dst;         /* [num_edges] */
    const float *edge_joint;          /* see "Layouts" */
    uint32_t joint_row_stride;        /* floats between rows of one table */
    uint64_t joint_edge_stride;       /* floats between consecutive edges' tables */
    /* optional CSR as in struct graph (node_list has num_nodes entries, the
     * last row ends at num_edges); NULL = stable sort by node, which is the
     * order set_up_*_nodes_to_edges produce */
    const uint32_t *dest_node_list, *dest_edge_list;
    const uint32_t *src_node_list, *src_edge_list;
    int32_t memory;                   /* bp_memory of every pointer above */
    int32_t flags;                    /* bp_graph_flags */
} bp_graph_desc;

typedef enum {
    /* renumber nodes internally by decreasing out-degree (ties by increasing
     * in-degree, then id) so the send buffers of frequent sources share
     * cache sectors and a warp's nodes have similar in-degrees; results are
     * unchanged (each node's in-edges keep their order), node ids at the API
     * stay the caller's.  Node-schedule loopy BP only: tree BP and the edge
     * schedule return BP_ERR_STATE on such a graph. */
    BP_GRAPH_REORDER_BY_OUT_DEGREE = 1
} bp_graph_flags;

typedef struct {
    float tolerance;          /* the reference's `convergence` */
    uint32_t max_iterations;
    uint32_t check_every;     /* 1: loopy_propagate_until[_edge]; 10 (BATCH_SIZE): the _acc variants */
    int32_t schedule;         /* bp_schedule */
    int32_t delta_mode;       /* bp_delta_mode */
    int32_t verbose;          /* print the reference's "No Convergence" line */
    uint32_t graph_chunk;     /* iterations per CUDA-graph launch; 0 = automatic */
    int32_t kernel_variant;   /* bp_kernel_variant of the node-schedule iteration kernel */
} bp_loopy_options;

typedef struct {
    uint32_t iterations;      /* the reference's return value */
    uint32_t executed;        /* iterations actually run */
    int32_t converged;        /* 1 when the stopping rule fired */
    float delta;              /* the reference's `delta` at return */
    float previous_delta;     /* the reference's `previous_delta` at return */
    double delta_f64;         /* f64 sum of the last check's |diff| terms */
    float elapsed_ms;         /* device time of the iteration loop */
    uint32_t serial_sums;     /* serial fp32 delta: serial sums formed because no
                               * bound decided the stop */
    uint32_t serial_refines;  /* serial fp32 delta: checks that needed the interval
                               * narrowed from the terms' own rounding errors */
    int32_t kernel_used;      /* bp_kernel_variant that ran the node-schedule
                               * iterations (block tiles for the one-launch loop
                               * of small graphs); 0 for the edge schedule */
} bp_loopy_result;

typedef struct {
    uint32_t num_levels;
    uint32_t num_waves;       /* kernel launches the forward + backward passes used */
    float elapsed_ms;
} bp_tree_result;

const char *bp_status_string(int status);
const char *bp_last_error(void);
int bp_version(void);

/* ---- graph lifetime -------------------------------------------------- */
int bp_graph_create(bp_graph **out, const bp_graph_desc *desc, void *stream);
void bp_graph_destroy(bp_graph *g);
int bp_graph_info(const bp_graph *g, uint32_t *num_nodes, uint32_t *num_edges,
                  uint32_t *max_states, uint32_t *uniform_states);
int bp_set_stream(bp_graph *g, void *stream);
int bp_synchronize(bp_graph *g);
/* bytes of device memory the graph holds */
int bp_graph_device_bytes(const bp_graph *g, uint64_t *bytes);
/* Graph buffers come from the current device's stream-ordered memory pool,
 * which this library sets to keep freed memory cached (so graph after graph
 * reuses it without cudaMalloc/cudaFree); this returns the cached memory to
 * the driver. */
int bp_release_cached_memory(void);
/* Grows that pool, once, to hold at least `bytes` (one block allocated and
 * freed at once), so that graphs built later carve their buffers out of the
 * reservation.  For serving loops that build and destroy graphs while others
 * solve: the pool otherwise grows in the middle of a build whenever no cached
 * block fits, and on a B200 such growth stalled a build (and a solve on
 * another stream) for up to a second.  No effect when the pool already holds
 * `bytes`; bp_release_cached_memory() gives the memory back. */
int bp_reserve_cached_memory(uint64_t bytes);

/* ---- state ----------------------------------------------------------- */
int bp_set_beliefs(bp_graph *g, const float *beliefs, uint32_t ld, int memory);
int bp_get_beliefs(bp_graph *g, float *beliefs, uint32_t ld, int memory);
/* the two message arrays: slot 0 and slot 1 (edges_messages and
 * last_edges_messages of struct graph); `latest` is the slot
 * *previous_edge_messages points at */
int bp_set_messages(bp_graph *g, int slot, const float *messages, uint32_t ld, int memory);
int bp_get_messages(bp_graph *g, int slot, float *messages, uint32_t ld, int memory);
int bp_set_latest_slot(bp_graph *g, int slot);
int bp_get_latest_slot(const bp_graph *g, int *slot);

/* ---- loopy BP -------------------------------------------------------- */
void bp_loopy_default_options(bp_loopy_options *opt);
/* init_previous_edge (graph.c:725-751): latest = normalise(J . belief_src) */
int bp_init_messages(bp_graph *g);
/* loopy_propagate_until / _edge / _acc / _edge_acc (graph.c:1186-1547) */
int bp_loopy(bp_graph *g, const bp_loopy_options *opt, bp_loopy_result *res);

/* The reference's serial fp32 delta sum (graph.c:1300-1309): *out = the sum
 * of the n non-negative DEVICE floats x[0..n) added one at a time in index
 * order in fp32, bit for bit, written to the DEVICE float *out on `stream`
 * (asynchronous).  Formed in parallel: inside one binade of the running sum
 * every add is the term rounded to that binade's unit, so a scan of
 * per-term increments gives the running sum exactly; a term that moves the
 * sum to the next binade is added alone.  method: 0 = 256 threads (the
 * form bp_loopy's final delta uses), 1 = 128 threads with 2048 floats of
 * staging (the iteration kernel's), 2 = 256 threads with 2048 floats,
 * 3 = the one-add-at-a-time chain, 4 = 1024 threads with 8192 floats. */
int bp_serial_sum_f32(const float *x, uint64_t n, float *out, int method, void *stream);
/* An interval [lohi[0], lohi[1]] (DEVICE doubles) holding that same serial
 * sum, narrowed from the terms' own rounding errors: exact for every add where
 * the running sum's binade is certain, half an ulp for the rest (binade
 * crossings, exact ties).  [0, +inf] when there is none (an inf term, or n
 * too large for the running bound). */
int bp_serial_sum_bounds(const float *x, uint64_t n, double *lohi, void *stream);

/* ---- one rank of a sharded loopy run --------------------------------- */
/* SURVEY's multi-GPU split of the node schedule (no counterpart in the
 * reference, which runs on one device): each rank (one process per GPU)
 * owns the destination nodes [node_begin, node_end) and holds their
 * in-edges (a bp_graph of all V nodes whose edges are those in-edges, built
 * from the full edge list filtered by destination, in edge order), every
 * node's beliefs, and two DEVICE send-buffer arrays of [V][max states]
 * floats.  Per iteration of loopy_propagate_until (graph.c:1278-1324):
 *   bp_flood_range reads every node's send buffer from q_in, writes the
 *     owned nodes' messages (into the slot after the latest one, which then
 *     becomes the latest), beliefs and next send buffers (q_out[node_begin,
 *     node_end)), and the f64 sum of the owned in-edges' |diff| terms to the
 *     DEVICE double *delta;
 *   the ranks then all-gather q_out and sum the deltas (every rank the same
 *     sum, in rank order) for the reference's stopping rule.
 * bp_send_buffers_range writes the first send buffers (read_incoming_messages,
 * graph.c:850-882, after init_previous_edge) of the owned nodes.  Results
 * are the single-GPU node schedule's bit for bit.  stream NULL = the graph's
 * stream.  Renumbered graphs return BP_ERR_STATE. */
int bp_send_buffers_range(bp_graph *g, uint32_t node_begin, uint32_t node_end, float *q_out, void *stream);
int bp_flood_range(bp_graph *g, uint32_t node_begin, uint32_t node_end, const float *q_in, float *q_out,
                   double *delta, void *stream);

/* ---- loopy BP without allocating ------------------------------------- */
/* No counterpart in the reference: an addition of this library.
 *
 * Who needs it: code that must not allocate GPU memory while it runs --
 * a host application that owns the device through its own allocator and
 * forbids components from calling cudaMalloc, a real-time loop that cannot
 * afford an allocation or the device-wide synchronisation cudaFree implies,
 * or a process pinned right at its memory cap.  This call runs the same
 * kernels as bp_loopy (node schedule, loopy_propagate_until semantics) and
 * allocates nothing: no cudaMalloc, no cudaFree, no allocating library
 * routine.
 *
 * Stopping rule: the reference's test (delta < tol or |delta - previous| <
 * tol, graph.c:1313) on a deterministic fp64 sum of the |diff| terms, i.e.
 * bp_loopy with BP_DELTA_F64.  It is NOT the reference's serial fp32 sum that
 * bp_loopy's default uses on small graphs: where delta or its step lies
 * within about 1e-4 relative of tol, the iteration count can differ by one
 * from the reference's.  Use bp_loopy with BP_DELTA_SERIAL_F32 when the
 * reference's exact decision is needed.  delta and previous_delta in the
 * result are that fp64 sum rounded to float.
 *
 * The caller passes every input and output as DEVICE memory, already in the
 * destination-sorted layout bp_graph_create builds internally:
 *   in_ptr   [num_nodes + 1]            row starts of each node's in-edges
 *   in_src   [num_edges]                source node of each position
 *   joint    [num_edges][S][S]          tables in position order
 *   beliefs  [num_nodes][S]             read and updated in place
 *   messages [2][num_edges][S]          the two message arrays; slot
 *                                       latest_slot holds the latest ones
 * with S = num_states for every node.  in_ptr and in_src are checked on the
 * device before anything reads through them (in_ptr[0] == 0, rows
 * non-decreasing, in_ptr[num_nodes] == num_edges, sources < num_nodes);
 * a violation returns BP_ERR_INVALID.  init_messages != 0 first fills the
 * latest slot with normalise(J . belief_src) (init_previous_edge), also when
 * max_iterations is 0.  On return *latest_out is the slot holding the newest
 * messages.
 *
 * Working memory (two send buffers of num_nodes * S floats, one double per
 * node tile, a control block) lives in one array of BP_NOALLOC_SCRATCH_BYTES
 * compiled into the library; every GPU that loads the library holds it until
 * the process exits.  Graphs whose working memory does not fit (about 1M
 * nodes at 2 states) are rejected with BP_ERR_SHAPE and a message giving the
 * size needed.
 *
 * Each call looks the array's device address up on the current device
 * (cudaGetSymbolAddress); the first call on a device also loads the module
 * there, so make that first call before any stream capture on the device.
 * All calls share the one array and leave their contents in it; each call
 * rewrites the control block and the buffers before reading them.  Calls
 * whose work overlaps on the GPU (other streams, other threads) race on
 * that array: serialise them. */
#define BP_NOALLOC_SCRATCH_BYTES (16u << 20)
int bp_loopy_noalloc(uint32_t num_nodes, uint32_t num_edges, uint32_t num_states,
                     const uint32_t *in_ptr, const uint32_t *in_src, const float *joint,
                     float *beliefs, float *messages, int latest_slot, int init_messages,
                     float tolerance, uint32_t max_iterations, void *stream,
                     bp_loopy_result *result, int *latest_out);

/* ---- tree BP --------------------------------------------------------- */
/* init_levels_to_nodes (graph.c:806-827); levels may be NULL (kept on device
 * side only), else receives 2*V entries in the reference's layout */
int bp_tree_build_levels(bp_graph *g, uint32_t *levels, uint32_t *num_levels);
/* use level lists computed elsewhere (struct graph's levels_to_nodes) */
int bp_tree_set_levels(bp_graph *g, const uint32_t *levels, uint32_t num_levels);
int bp_tree_start(bp_graph *g);                       /* graph.c:376-424 */
int bp_tree_level(bp_graph *g, uint32_t level);       /* graph.c:524-538 */
int bp_tree_reset_visited(bp_graph *g);               /* graph.c:598-605 */
int bp_tree_marginalize(bp_graph *g);                 /* graph.c:588-596 */
/* the whole driver sequence (c_benchmark/main.c:224-236) in one call */
int bp_tree(bp_graph *g, bp_tree_result *res);
int bp_set_visited(bp_graph *g, const char *visited); /* host [V] */
int bp_get_visited(bp_graph *g, char *visited);       /* host [V] */

/* ---- batched loopy BP -------------------------------------------------- */
/* Many independent networks, each with its own stopping rule
 * (loopy_propagate_until per network), solved in one persistent launch per
 * state count: a thread block takes the next network from a work queue
 * (largest first) and iterates it to convergence.  Each network's result is
 * what bp_loopy gives for it alone.  Every node of one network has the same
 * state count; networks may differ.
 *
 * Layout of the batch-wide arrays (bp_batch_layout): network n's beliefs are
 * [V_n][S_n] floats at belief_offsets[n], its messages [E_n][S_n] (edge-id
 * order) at message_offsets[n]; offsets[N] is the total.  Offsets are
 * multiples of 4 floats; the gaps between networks are padding. */
typedef struct bp_batch bp_batch;

typedef struct {
    float tolerance;          /* per network, the reference's `convergence` */
    uint32_t max_iterations;  /* per network */
    int32_t delta_mode;       /* BP_DELTA_F64 (default) or BP_DELTA_SERIAL_F32 */
    uint32_t block_threads;   /* threads per network block; 0 = as tuned (bp_batch_autotune) */
    int32_t init_messages;    /* 1: init_previous_edge first */
    int32_t reserved;
} bp_batch_options;

typedef struct {
    uint32_t num_networks;
    uint32_t converged;       /* networks whose stopping rule fired */
    uint32_t max_executed;    /* most iterations any network ran */
    float elapsed_ms;         /* device time of the batched solve */
} bp_batch_result;

/* descs: one bp_graph_desc per network, host memory */
int bp_batch_create(bp_batch **out, uint32_t num_networks, const bp_graph_desc *descs, void *stream);
void bp_batch_destroy(bp_batch *b);
int bp_batch_layout(const bp_batch *b, uint64_t *belief_offsets, uint64_t *message_offsets);
/* setting beliefs marks slot 1 as the latest messages of every network, as
 * create_graph leaves struct graph */
int bp_batch_set_beliefs(bp_batch *b, const float *beliefs, int memory);
int bp_batch_get_beliefs(bp_batch *b, float *beliefs, int memory);
int bp_batch_get_messages(bp_batch *b, float *messages, int memory);
void bp_batch_default_options(bp_batch_options *o);
/* The networks are grouped by state count; with BP_BATCH_SMALL_NODES=n
 * (environment, read at create; default 0 = off) the networks of at most n
 * nodes of a state count form a group of their own, with its own launch
 * shape, work queue and stream.
 * bp_batch_autotune times 64/128/256/512 threads per network block, and
 * blocks in flight, for each group on this batch, keeps the fastest (results
 * cached in $BP_AUTOTUNE_CACHE, default ~/.cache/bp_b200_autotune.txt);
 * beliefs and messages are restored */
int bp_batch_autotune(bp_batch *b, const bp_batch_options *o);
/* per group (at most *count entries; *count returns the number of groups):
 * its state count and threads per block (a state count appears once per size
 * class) */
int bp_batch_get_block_threads(const bp_batch *b, uint32_t *states, uint32_t *block, uint32_t *count);
/* per group as above, plus max_nodes: the group's size bound (0 = none, the
 * group of larger networks) and grid: its blocks in flight */
int bp_batch_get_groups(const bp_batch *b, uint32_t *states, uint32_t *max_nodes, uint32_t *block, uint32_t *grid,
                        uint32_t *count);
/* the whole batch: one CUDA graph launch */
int bp_batch_loopy(bp_batch *b, const bp_batch_options *o, bp_batch_result *r);
int bp_batch_network_results(bp_batch *b, uint32_t *iterations, uint32_t *executed, int32_t *converged,
                             float *delta);

/* ---- differentiable unrolled loopy BP --------------------------------- */
/* T synchronous iterations of the reference's update on a pairwise model:
 * priors softmax(log_unary[v]), joint tables exp(log_pair[k]) shared by the
 * edges that name table k (edge_table[e] & 0x7f; bit 0x80 = the edge uses
 * the transposed table).  The iteration runs in the log domain (the
 * reference's update multiplies each belief into itself every iteration, so
 * beliefs head to 0 faster than fp32 can follow in linear form).
 * bp_unrolled_forward writes the LOG-beliefs after T iterations;
 * bp_unrolled_backward maps d loss / d log-beliefs to gradients with respect
 * to log_unary and log_pair with a hand-written adjoint.  The forward keeps
 * the iteration state every checkpoint_every iterations; the backward
 * recomputes each segment from its checkpoint.  With one table and at most
 * 8 states the adjoint runs in pull form (each source gathers its
 * out-neighbours' message adjoints; BP_UBWD_PULL=0 selects the scatter form
 * at create, which every other shape uses).  Tensor arguments of
 * forward/backward are device memory, 16-byte aligned; the graph arrays of
 * create are host memory.  At most 16 tables. */
typedef struct bp_unrolled bp_unrolled;
/* Cross-entropy loss head for the unrolled engine's log-beliefs: on `stream`,
 * *loss (a DEVICE float) = -(1/V) sum_v log_beliefs[v*S + labels[v]], summed
 * in f64 in a fixed order; scratch: 297 DEVICE doubles, zeroed before the
 * first call (the last block resets the ticket it keeps there).
 * bp_nll_grad_f32 writes the gradient: grad_log_beliefs[v*S + s] =
 * -grad_loss[0] / V at s == labels[v], else 0 (grad_loss a DEVICE float).
 * A label outside [0, S) makes the loss NaN. */
int bp_nll_f32(const float *log_beliefs, const int64_t *labels, uint32_t V, uint32_t S, double *scratch,
               float *loss, void *stream);
int bp_nll_grad_f32(const int64_t *labels, uint32_t V, uint32_t S, const float *grad_loss, float *grad_log_beliefs,
                    void *stream);

int bp_unrolled_create(bp_unrolled **out, uint32_t num_nodes, uint32_t num_edges, uint32_t num_states,
                       uint32_t num_tables, const uint32_t *edge_src, const uint32_t *edge_dst,
                       const uint8_t *edge_table, uint32_t iterations, uint32_t checkpoint_every,
                       void *stream);
void bp_unrolled_destroy(bp_unrolled *u);
int bp_unrolled_set_stream(bp_unrolled *u, void *stream);
int bp_unrolled_forward(bp_unrolled *u, const float *log_unary, const float *log_pair, float *log_beliefs);
int bp_unrolled_backward(bp_unrolled *u, const float *grad_log_beliefs, float *grad_log_unary,
                         float *grad_log_pair);

/* ---- drop-in support (struct graph from graph.h) ---------------------- */
struct graph;
int bp_set_sync_mode(struct graph *g, int mode);
int bp_sync_host(struct graph *g);
/* the device mirror of a struct graph, creating it if needed */
int bp_graph_of(struct graph *g, bp_graph **out);

#ifdef __cplusplus
}
#endif

#endif /* BP_H_ */
