// bp_internal.h -- device-resident graph shared by the engine's .cu files.
//
// HBM layout (one graph, S_max states, "position" = index in the
// destination-sorted edge order, i.e. the reference's dest_nodes_to_edges
// order, graph.c:285-313):
//
//   in_ptr   u32 [V+1]        row starts of each node's in-edges
//   in_src   u32 [E]          source node of the edge at position p
//   pos_edge u32 [E]          edge id at position p      (dest_nodes_to_edges_edge_list)
//   edge_pos u32 [E]          position of edge id e (built on first use)
//   pos_dims u8  [E]          x | y<<4 (source / destination state count); mixed graphs only
//   node_s   u8  [V]          state count per node; mixed graphs only
//   joint    f32 [E][MS][MS]  joint tables in position order, zero padded
//   belief   f32 [V][MS]      beliefs, zero beyond S_v
//   msg[2]   f32 [E][MS]      the two message arrays (struct graph's
//                             edges_messages / last_edges_messages), position order
//   q[2]     f32 [V][MS]      send buffers of the fused flooding schedule
//
// Messages are stored by destination so a node's incoming messages are one
// contiguous run: the gather needs no atomics and reads whole sectors.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <chrono>

#include <nvtx3/nvToolsExt.h>

#include "bp.h"

namespace bpx {

constexpr int kMaxStates = BP_MAX_STATES;
// allocated entries past the ends of in_ptr and belief (nodes) and of
// in_src, joint and msg (edges): the staged iteration kernel copies whole
// node tiles and 16-byte-rounded ranges
constexpr uint32_t kArrayPadNodes = 264;
constexpr uint32_t kArrayPadEdges = 8;

// Control block of one loopy run, resident in device memory.  Kernels read it
// at entry (iteration index, buffer parities, stop flag) and the last block
// of each iteration updates it, so a CUDA graph of identical launches can run
// the whole loop with the reference's stopping rule evaluated on the device.
struct LoopyCtl {
    uint32_t it;           // iterations executed so far in this run
    uint32_t done;         // 0 running, 1 stopping rule fired, 2 ran out of iterations, 3 a device wait timed out
    uint32_t ret;          // the reference's return value
    uint32_t counter;      // last-block-done ticket
    uint32_t num_iter;     // _acc variants: completed batches * check_every
    uint32_t final_i;      // the reference's loop variable at exit
    uint32_t max_it;
    uint32_t check_every;
    uint32_t msg_parity0;  // slot holding the latest messages when the run started
    uint32_t q_parity0;
    uint32_t serial;       // 1 = serial fp32 delta kernel decides
    uint32_t acc_edge;     // edge schedule, _acc variant
    float tol;
    float delta_f, prev_f;
    uint32_t pad0;
    double delta_d, prev_d;
    // grid barrier of the fused (one-launch) loop: arrivals, generation, and
    // a flag a block sets when its bounded wait ran out
    uint32_t bar_count, bar_gen, bar_fail;
    // test hook of that bounded wait (BP_DEBUG_BARRIER_SKIP): block
    // bar_skip - 1 does not arrive at the first barrier, so the others' waits
    // run out; 0 = off
    uint32_t bar_skip;
    // serial mode: the reference's fp32 sum of a check's |diff| terms lies
    // in [dlo, dhi] (f64 sum of the terms +- the serial sum's rounding bound),
    // and in [plo, phi] for the previous check; *_exact = the serial sum
    // itself was formed (lo == hi == the float).  The terms of each check go
    // to buffer (check index % 3) of absdiff, ad_stride floats apart.
    uint64_t n_terms, ad_stride;
    double dlo, dhi, plo, phi;
    uint32_t delta_exact, prev_exact, cur_buf, prev_buf;
    uint32_t serial_sums;  // serial sums formed because the bound could not decide
    // the one-launch loop: block 0's serial sums for the other blocks
    uint32_t fb_pform;     // the previous delta was formed too
    float fb_s, fb_p;
    // [dlo, dhi] / [plo, phi] narrowed from the terms' own rounding errors
    uint32_t delta_ref, prev_ref;
    uint32_t serial_refines;   // checks that needed the narrowed interval
    uint32_t wait_ms;          // limit of the grid barrier's wait; 0 = 2000 ms
};

struct TreeData {
    bool ready = false;
    uint32_t num_levels = 0;
    uint32_t *levels_host = nullptr;   // copy of the level lists (2V)
    // per node: level and index within level (host + device)
    uint32_t *d_node_level = nullptr, *d_node_lidx = nullptr;
    // waves: nodes of each (level, wave) contiguous
    uint32_t *d_wave_nodes = nullptr;
    uint32_t *wave_off = nullptr;      // host [num_waves_total + 1]
    uint32_t *level_wave_begin = nullptr; // host [num_levels + 1] index into waves
    uint32_t total_waves = 0;
    cudaGraphExec_t exec = nullptr;    // bp_tree's launch sequence, captured once
    // schedule order: k = a node's index in d_wave_nodes.  Per k (s_*), and
    // per out-edge with the out-edges grouped by their source's k (q order,
    // q_*), so the nodes of a wave read their records and out-edges as
    // contiguous runs:
    uint2 *s_in = nullptr;             // [V] in-edge range (positions) of node k
    uint32_t *s_out = nullptr;         // [V + 1] out-edge range of node k in q order
    uint32_t *s_lidx = nullptr;        // [V] index in its level
    uint8_t *s_S = nullptr;            // [V] state count
    float *q_joint = nullptr;          // x-by-y tables (row stride y), each padded to 4 floats
    uint32_t *q_joff = nullptr;        // [E] float offset of out-edge q's table
    uint2 *q_lvidx = nullptr;          // [E] (level, index in level) of out-edge q's destination
    uint8_t *q_y = nullptr;            // [E] state count of out-edge q's destination
    uint32_t *q_pos = nullptr;         // [E] message position of out-edge q
    uint32_t *q_dst = nullptr;         // [E] destination of out-edge q
    uint32_t *d_wave_off = nullptr;    // device copy of wave_off (the cooperative tail launches)
    uint32_t *d_bar = nullptr;         // grid barrier of a tail launch: arrivals, generation, failure
};

}  // namespace bpx

struct bp_graph {
    uint32_t V = 0, E = 0;
    uint32_t ms = 1;         // storage stride = max state count
    uint32_t uniform = 0;    // common state count, or 0 when mixed
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    uint32_t *in_ptr = nullptr, *in_src = nullptr, *pos_edge = nullptr, *edge_pos = nullptr;
    // node renumbering (BP_GRAPH_REORDER_BY_OUT_DEGREE): internal id i holds the
    // caller's node new_to_old[i]; null when ids are the caller's
    uint32_t *new_to_old = nullptr;
    // renumbered graphs: internal ids below this have two or more out-edges
    uint32_t reuse_nodes = 0;
    uint8_t *pos_dims = nullptr, *node_s = nullptr;
    float *joint = nullptr;
    float *belief = nullptr;
    float *msg[2] = {nullptr, nullptr};
    float *q[2] = {nullptr, nullptr};
    int latest = 0;

    // Split flooding schedule (loopy.cu, layout built by engine.cu): the
    // edges again in "send order" -- grouped by the range of their source
    // node (range_nodes consecutive ids per range, so one range's send
    // buffers fit L2), in position order inside a range.  The send pass reads
    // these streams contiguously and gathers Q from one range at a time; the
    // node pass reads each in-edge's message through s_inv.
    struct Split {
        int state = 0;                   // 0 not built, 1 ready, -1 not applicable to this graph
        uint32_t R = 0;                  // source ranges
        uint32_t range_nodes = 0;
        uint32_t *s_src = nullptr;       // [E] source node (send order)
        uint32_t *s_edge = nullptr;      // [E] edge id (serial delta terms)
        uint32_t *s_pos = nullptr;       // [E] position of send index k
        uint32_t *s_inv = nullptr;       // [E] send index of position p
        float *s_joint = nullptr;        // [E][MS][MS]
        float *s_msg[2] = {nullptr, nullptr};   // the two message arrays in send order
    } split;

    // src-CSR, built on first use (tree schedule)
    uint32_t *out_ptr = nullptr, *out_pos = nullptr, *out_dst = nullptr, *pos_dst = nullptr;

    // scratch
    double *partials = nullptr;
    uint32_t partials_cap = 0;
    float *absdiff = nullptr;
    bpx::LoopyCtl *ctl = nullptr;
    bpx::LoopyCtl *ctl_host = nullptr;   // pinned
    uint8_t *visited = nullptr;
    float *staging = nullptr;
    size_t staging_bytes = 0;

    // host-side copies of small structure arrays (tree waves, edge-variant runs)
    uint8_t *node_s_host = nullptr;      // [V] state counts
    uint32_t *in_ptr_host = nullptr;     // [V+1], on demand
    uint32_t *run_len = nullptr;         // [nruns] runs of equal state count (device)
    uint8_t *run_s = nullptr;
    uint32_t nruns = 0;

    bpx::TreeData tree;

    // cached CUDA graphs of the iteration loop
    struct CachedGraph {
        cudaGraphExec_t exec = nullptr;
        uint64_t key = 0;
    } loop_graph[4];

    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint64_t device_bytes = 0;
};

namespace bpx {

// error plumbing (engine.cu)
int set_error(int status, const char *fmt, ...);
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define BP_CUDA(call)                                                      \
    do {                                                                   \
        cudaError_t e_ = (call);                                           \
        if (e_ != cudaSuccess) return bpx::cuda_fail(e_, #call, __FILE__, __LINE__); \
    } while (0)

int dev_alloc(bp_graph *g, void **p, size_t bytes);
// tree schedule (tree.cu, levels_gpu.cu)
void tree_clear(bp_graph *g);
int tree_prepare_host(bp_graph *g, const uint32_t *levels, uint32_t num_levels);
int tree_build_levels_gpu(bp_graph *g, uint32_t *levels, uint32_t *num_levels);
int ensure_staging(bp_graph *g, size_t bytes);
int ensure_edge_pos(bp_graph *g);
int ensure_out_csr(bp_graph *g);
int ensure_host_in_ptr(bp_graph *g);
// split flooding schedule: build g->split with source ranges of
// `range_nodes` ids (uniform graphs of at most 4 states; else state -1)
void split_free(bp_graph *g);
int split_build(bp_graph *g, uint32_t range_nodes);
// the split layout for a graph the default loop runs split (loopy.cu)
int flood_split_prepare(bp_graph *g);

// an NVTX range for the lifetime of the object: the entry points show up
// as named ranges on a profiler's timeline (no cost without a tool attached)
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// BP_TRACE=1: wall time of each stage of a multi-stage call on stderr (each
// mark waits for the graph's stream, so tracing serialises the stages); the
// call is an NVTX range and each stage an NVTX mark in any case
struct StageTrace {
    bool on;
    cudaStream_t s;
    const char *what;
    std::chrono::steady_clock::time_point t;
    NvtxRange range;
    StageTrace(cudaStream_t s_, const char *what_)
        : on(getenv("BP_TRACE") != nullptr), s(s_), what(what_), t(std::chrono::steady_clock::now()), range(what_) {}
    void mark(const char *stage) {
        nvtxMarkA(stage);
        if (!on) return;
        cudaStreamSynchronize(s);
        const auto n = std::chrono::steady_clock::now();
        fprintf(stderr, "bp_trace %s %-22s %9.3f ms\n", what, stage,
                std::chrono::duration<double, std::milli>(n - t).count());
        t = n;
    }
};

inline unsigned grid_for(uint64_t n, unsigned block) {
    uint64_t b = (n + block - 1) / block;
    if (b == 0) b = 1;
    if (b > 0x7fffffffull) b = 0x7fffffffull;
    return (unsigned)b;
}

}  // namespace bpx
