// tree.cu -- tree BP as level-synchronous frontier passes.
//
// The reference's schedule (c_benchmark/main.c:224-236):
//   propagate_using_levels_start   level 0 sends its beliefs on every out-edge
//   propagate_using_levels(l)      l = 1 .. L-2, then (after reset_visited)
//                                  l = L-1 .. 1: each node of the level, in
//                                  order, marks itself visited, multiplies its
//                                  incoming messages (no prior) and sends to
//                                  the out-neighbours not yet visited
//   marginalize                    belief = normalise(prod of incoming messages)
// A level is split into waves (levels.c); one wave is one launch of
// k_tree_wave with a thread per node.  "Not yet visited" at node u's turn is
//   visited-before-this-call[w]  or  (w in this level and index(w) <= index(u)),
// which is what the sequential loop sees, so any call order the reference
// accepts gives the reference's messages.  All messages live in slot 0
// (struct graph's edges_messages), position order.
#include <cub/device/device_scan.cuh>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "bp_device.cuh"
#include "bp_internal.h"
#include "bp_levels.h"

namespace bpx {

// Schedule order.  The nodes are listed wave by wave, level by level
// (TreeData::d_wave_nodes); a node's index k in that list is its schedule
// index, and a wave is a range of k.  Per node the kernels read records in
// schedule order (TreeData::s_*: in-edge range, out-edge range, index in
// level, state count), so the threads of a wave read them as contiguous
// runs, and the out-edges are laid out by the source's schedule index
// (TreeData::q_*: message position, destination, destination level data and
// state count, dense table), so a wave's out-edge data is one contiguous
// stream.  The random accesses left are the incoming messages, the message
// stores (both in position order) and, at level 0, the beliefs.
//
// Who has been visited.  The graph.h calls keep the visited flags in
// g->visited (mode 0).  bp_tree runs the whole schedule from cleared flags,
// so the flags at node u's turn in level l are a function of the levels:
// upward (mode 1) every node of a level below l, downward (mode 2) every node
// of a level above l, and in both the nodes of l up to u's index; bp_tree
// reads no flags and writes the final ones (levels >= 1) once at the end.

struct TreeArgs {
    const uint32_t *nodes;            // schedule order -> node
    const uint2 *s_in;                // [k] in-edge range (positions) of node k
    const uint32_t *s_out;            // [k], [k + 1]: out-edge range (q order)
    const uint32_t *s_lidx;           // [k] index in its level
    const uint8_t *s_S;               // [k] state count
    const uint32_t *q_pos, *q_dst;    // [q] message position, destination
    const uint2 *q_lvidx;             // [q] destination (level, index in level)
    const uint8_t *q_y;               // [q] destination state count
    const uint32_t *q_joff;           // [q] offset of the dense table in q_joint
    const float *q_joint;
    const float *belief;
    float *msg;
    uint8_t *visited;
};

// has w (out-edge q, level data li) been visited at the turn of the node
// with index my_idx in `level`?
__device__ __forceinline__ bool tree_seen(const TreeArgs &a, int mode, uint32_t level, uint32_t my_idx, uint32_t q,
                                          uint2 li) {
    const bool earlier = li.x == level && li.y <= my_idx;
    if (mode == 1) return li.x < level || earlier;
    if (mode == 2) return li.x > level || earlier;
    return a.visited[a.q_dst[q]] || earlier;
}

// propagate_using_levels_start (graph.c:376-424): level 0 is schedule
// indices [k0, k0 + n); mark: set the visited flags (graph.h calls)
template <int MS, bool UNI>
__global__ void k_tree_start(const TreeArgs a, uint32_t k0, uint32_t n, int mark) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const uint32_t k = k0 + t;
    const uint32_t u = a.nodes[k];
    if (mark) a.visited[u] = 1;
    const int x = UNI ? MS : a.s_S[k];
    float buf[MS];
    ldv<MS>(a.belief + (size_t)u * MS, buf);
    for (uint32_t q = a.s_out[k]; q < a.s_out[k + 1]; ++q) {
        const uint32_t p = a.q_pos[q];
        const int y = UNI ? MS : a.q_y[q];
        float m[MS];
        send_msg_dense<MS, UNI>(a.q_joint + a.q_joff[q], buf, x, y, m);
        stv<MS>(a.msg + (size_t)p * MS, m);
    }
}

// one wave of propagate_node_using_levels (graph.c:461-522): schedule
// indices [k0, k0 + n) of `level`, a thread per node
template <int MS, bool UNI>
__global__ void k_tree_wave(const TreeArgs a, uint32_t k0, uint32_t n, uint32_t level, int mode) {
    griddep_launch_dependents();
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    // the schedule's records first (no tree kernel writes them), then the
    // wait for the kernels ahead, whose messages and visited flags follow
    const uint32_t k = k0 + t;
    const int S = UNI ? MS : a.s_S[k];
    const uint32_t my_idx = a.s_lidx[k];
    const uint2 r = a.s_in[k];
    const uint32_t o0 = a.s_out[k], o1 = a.s_out[k + 1];
    griddep_wait();
    float buf[MS];
#pragma unroll
    for (int i = 0; i < MS; ++i) buf[i] = (UNI || i < S) ? 1.0f : 0.0f;
    for (uint32_t p = r.x; p < r.y; ++p) {
        float mm[MS];
        ldv<MS>(a.msg + (size_t)p * MS, mm);
        combine<MS, UNI>(buf, mm, S);
    }
    for (uint32_t q = o0; q < o1; ++q) {
        if (tree_seen(a, mode, level, my_idx, q, a.q_lvidx[q])) continue;
        const uint32_t p = a.q_pos[q];
        const int y = UNI ? MS : a.q_y[q];
        float m[MS];
        send_msg_dense<MS, UNI>(a.q_joint + a.q_joff[q], buf, S, y, m);
        stv<MS>(a.msg + (size_t)p * MS, m);
    }
}

// the same step with a group of G lanes (2 .. 32) per node, for waves too
// small to fill the GPU with a thread per node (their time is one node's chain
// of dependent loads): the lanes load G incoming messages at a time and every
// lane multiplies them into the buffer in edge order (shuffled from the
// loading lane), so the product is the thread-per-node one bit for bit; the
// sends to the out-neighbours go out in parallel, one per lane.  A group's
// lanes share the node, hence its trip counts, so the group mask is converged.
template <int MS, bool UNI, int G>
__global__ void k_tree_wave_group(const TreeArgs a, uint32_t k0, uint32_t n, uint32_t level, int mode) {
    static_assert(G >= 2 && G <= 32 && (G & (G - 1)) == 0, "group of 2..32 lanes");
    const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) / G;
    const uint32_t lane = threadIdx.x & (G - 1);
    const uint32_t gmask = G == 32 ? 0xffffffffu : (((1u << G) - 1u) << ((threadIdx.x & 31) & ~(G - 1)));
    griddep_launch_dependents();
    if (t >= n) return;   // the whole group
    // the schedule's records first (no tree kernel writes them): the node's
    // ranges, and this lane's first out-edge with its destination's level data
    // and table (into L2 for the latency-bound small waves); then the wait
    // for the kernels ahead, whose messages and visited flags follow
    const uint32_t k = k0 + t;
    const int S = UNI ? MS : a.s_S[k];
    const uint32_t my_idx = a.s_lidx[k];
    const uint2 r = a.s_in[k];
    const uint32_t o0 = a.s_out[k], o1 = a.s_out[k + 1];
    const uint32_t q0 = o0 + lane;
    uint32_t pp0 = 0, jo0 = 0;
    uint2 li0 = make_uint2(0u, 0u);
    int y0 = MS;
    if (q0 < o1) {
        pp0 = a.q_pos[q0];
        li0 = a.q_lvidx[q0];
        jo0 = a.q_joff[q0];
        if (!UNI) y0 = a.q_y[q0];
        if constexpr (G >= 16) {
            const float *jt = a.q_joint + jo0;
            prefetch_l2(jt);
            if constexpr (MS * MS > 32) prefetch_l2(jt + 32);
        }
    }
    griddep_wait();
    float buf[MS];
#pragma unroll
    for (int i = 0; i < MS; ++i) buf[i] = (UNI || i < S) ? 1.0f : 0.0f;
    for (uint32_t p0 = r.x; p0 < r.y; p0 += G) {
        float mm[MS];
#pragma unroll
        for (int i = 0; i < MS; ++i) mm[i] = 0.0f;
        if (p0 + lane < r.y) ldv<MS>(a.msg + (size_t)(p0 + lane) * MS, mm);
        const uint32_t cnt = min((uint32_t)G, r.y - p0);
        for (uint32_t j = 0; j < cnt; ++j) {
            float mj[MS];
#pragma unroll
            for (int i = 0; i < MS; ++i) mj[i] = __shfl_sync(gmask, mm[i], (int)j, G);
            combine<MS, UNI>(buf, mj, S);
        }
    }
    for (uint32_t q = q0; q < o1; q += G) {
        const bool first = q == q0;
        if (tree_seen(a, mode, level, my_idx, q, first ? li0 : a.q_lvidx[q])) continue;
        const uint32_t p = first ? pp0 : a.q_pos[q];
        const int y = UNI ? MS : (first ? y0 : (int)a.q_y[q]);
        float m[MS];
        send_msg_dense<MS, UNI>(a.q_joint + (first ? jo0 : a.q_joff[q]), buf, S, y, m);
        stv<MS>(a.msg + (size_t)p * MS, m);
    }
}

// ---- the small waves of a level in one cooperative launch ---------------
// A level's run of consecutive small waves (a warp per node) is one launch
// whose blocks meet at a grid barrier between waves, instead of one launch
// per wave: each such wave is a chain of a few dependent loads, so the
// launch between two waves cost as much as the wave.  Messages written by a
// wave are read by the next ones through L2 (ld.cg), since another SM may
// hold a stale line in L1.  The barrier's wait is bounded (2 s); a block
// whose wait runs out sets bar[2] and leaves, and the others leave at their
// next barrier; bp_tree then returns BP_ERR_TIMEOUT.
struct TreeTailArgs {
    TreeArgs t;
    const uint32_t *wave_off;
    uint32_t w0, w1, level;
    int mode;
    uint32_t *bar;   // arrivals, generation, failure flag (zeroed before the launch)
};

constexpr uint64_t kTailWaitNs = 2000000000ull;

__device__ __forceinline__ bool tail_barrier(uint32_t *bar, uint32_t &gen, uint32_t *s_fail) {
    __syncthreads();
    if (threadIdx.x == 0 && !*s_fail) {
        const uint32_t g0 = gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            bar[0] = 0;
            __threadfence();
            atomicExch(bar + 1, g0 + 1u);
        } else {
            const uint64_t t0 = global_ns();
            while (*(volatile uint32_t *)(bar + 1) == g0) {
                if (global_ns() - t0 > kTailWaitNs || *(volatile uint32_t *)(bar + 2)) {
                    *s_fail = 1;
                    atomicExch(bar + 2, 1u);
                    break;
                }
                __nanosleep(32);
            }
        }
        __threadfence();
    }
    __syncthreads();
    gen += 1;
    return *s_fail == 0;
}

// the node with schedule index k of a wave with a warp (k_tree_wave_group's
// step, G = 32, the incoming messages read through L2)
template <int MS, bool UNI>
__device__ __forceinline__ void tail_node(const TreeTailArgs &ta, uint32_t k, uint32_t lane) {
    const TreeArgs &a = ta.t;
    const int S = UNI ? MS : a.s_S[k];
    const uint32_t my_idx = a.s_lidx[k];
    const uint2 r = a.s_in[k];
    const uint32_t o0 = a.s_out[k], o1 = a.s_out[k + 1];
    float buf[MS];
#pragma unroll
    for (int i = 0; i < MS; ++i) buf[i] = (UNI || i < S) ? 1.0f : 0.0f;
    for (uint32_t p0 = r.x; p0 < r.y; p0 += 32) {
        float mm[MS];
#pragma unroll
        for (int i = 0; i < MS; ++i) mm[i] = 0.0f;
        if (p0 + lane < r.y) {
#pragma unroll
            for (int i = 0; i < MS; ++i) mm[i] = __ldcg(a.msg + (size_t)(p0 + lane) * MS + i);
        }
        const uint32_t cnt = min(32u, r.y - p0);
        for (uint32_t j = 0; j < cnt; ++j) {
            float mj[MS];
#pragma unroll
            for (int i = 0; i < MS; ++i) mj[i] = __shfl_sync(0xffffffffu, mm[i], (int)j);
            combine<MS, UNI>(buf, mj, S);
        }
    }
    for (uint32_t q = o0 + lane; q < o1; q += 32) {
        if (tree_seen(a, ta.mode, ta.level, my_idx, q, a.q_lvidx[q])) continue;
        const uint32_t p = a.q_pos[q];
        const int y = UNI ? MS : (int)a.q_y[q];
        float m[MS];
        send_msg_dense<MS, UNI>(a.q_joint + a.q_joff[q], buf, S, y, m);
        stv<MS>(a.msg + (size_t)p * MS, m);
    }
}

template <int MS, bool UNI>
__global__ void __launch_bounds__(256) k_tree_tail(const TreeTailArgs a) {
    __shared__ uint32_t s_fail;
    if (threadIdx.x == 0) s_fail = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    uint32_t gen = 0;
    for (uint32_t w = a.w0; w < a.w1; ++w) {
        const uint32_t lo = a.wave_off[w], n = a.wave_off[w + 1] - lo;
        for (uint32_t k = warp; k < n; k += nwarps) tail_node<MS, UNI>(a, lo + k, lane);
        if (w + 1 < a.w1 && !tail_barrier(a.bar, gen, &s_fail)) return;
    }
}

// ---- the schedule-order arrays (TreeData::s_*, q_*) -----------------------
// per schedule index: the node's in-edge range, index in level, state count
// and out-degree (scanned into s_out)
__global__ void k_ts_nodes(uint32_t V, const uint32_t *__restrict__ nodes, const uint32_t *__restrict__ in_ptr,
                           const uint32_t *__restrict__ out_ptr, const uint32_t *__restrict__ node_lidx,
                           const uint8_t *__restrict__ node_s, uint2 *__restrict__ s_in, uint32_t *__restrict__ s_lidx,
                           uint8_t *__restrict__ s_S, uint32_t *__restrict__ deg) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= V) return;
    const uint32_t u = nodes[k];
    s_in[k] = make_uint2(in_ptr[u], in_ptr[u + 1]);
    s_lidx[k] = node_lidx[u];
    s_S[k] = node_s[u];
    deg[k] = out_ptr[u + 1] - out_ptr[u];
}

// per out-edge in q order: the destination's state count and the padded
// table size
__global__ void k_tq_sizes(uint32_t V, const uint32_t *__restrict__ nodes, const uint32_t *__restrict__ s_out,
                           const uint32_t *__restrict__ out_ptr, const uint32_t *__restrict__ out_dst,
                           const uint8_t *__restrict__ node_s, uint8_t *__restrict__ q_y,
                           uint32_t *__restrict__ size) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= V) return;
    const uint32_t u = nodes[k], x = node_s[u], e0 = out_ptr[u], q0 = s_out[k], n = s_out[k + 1] - q0;
    for (uint32_t j = 0; j < n; ++j) {
        const uint32_t y = node_s[out_dst[e0 + j]];
        q_y[q0 + j] = (uint8_t)y;
        size[q0 + j] = (x * y + 3u) & ~3u;
    }
}

// the dense tables (rows of y floats, zero padding), message positions,
// destinations and the destinations' (level, index in level)
template <int MS>
__global__ void k_tq_fill(uint32_t V, const uint32_t *__restrict__ nodes, const uint32_t *__restrict__ s_out,
                          const uint32_t *__restrict__ out_ptr, const uint32_t *__restrict__ out_pos,
                          const uint32_t *__restrict__ out_dst, const uint8_t *__restrict__ node_s,
                          const uint8_t *__restrict__ q_y, const uint32_t *__restrict__ q_joff,
                          const float *__restrict__ joint, const uint32_t *__restrict__ node_level,
                          const uint32_t *__restrict__ node_lidx, float *__restrict__ q_joint,
                          uint2 *__restrict__ q_lvidx, uint32_t *__restrict__ q_pos, uint32_t *__restrict__ q_dst) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= V) return;
    const uint32_t u = nodes[k], x = node_s[u], e0 = out_ptr[u], q0 = s_out[k], n = s_out[k + 1] - q0;
    for (uint32_t j = 0; j < n; ++j) {
        const uint32_t q = q0 + j, y = q_y[q], p = out_pos[e0 + j], w = out_dst[e0 + j];
        float *dst = q_joint + q_joff[q];
        const float *src = joint + (size_t)p * (MS * MS);
        for (uint32_t i = 0; i < x; ++i)
            for (uint32_t c = 0; c < y; ++c) dst[i * y + c] = src[i * MS + c];
        for (uint32_t c = x * y; c < ((x * y + 3u) & ~3u); ++c) dst[c] = 0.0f;
        q_lvidx[q] = make_uint2(node_level[w], node_lidx[w]);
        q_pos[q] = p;
        q_dst[q] = w;
    }
}

__global__ void k_mark_visited(const uint32_t *__restrict__ nodes, uint32_t n, uint8_t *__restrict__ visited) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) visited[nodes[k]] = 1;
}

// the flags the whole schedule leaves: cleared before the downward pass,
// then set for every node of levels L-1 .. 1
__global__ void k_final_visited(uint32_t V, const uint32_t *__restrict__ node_level, uint8_t *__restrict__ visited) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < V) visited[v] = node_level[v] >= 1u ? 1 : 0;
}

// marginalize (graph.c:540-596): the belief is replaced by the product of
// the incoming messages when there is one, then normalised
template <int MS, bool UNI>
__global__ void k_tree_marginalize(uint32_t V, const uint32_t *__restrict__ in_ptr, const uint8_t *__restrict__ node_s,
                                   const float *__restrict__ msg, float *__restrict__ belief) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int S = UNI ? MS : node_s[v];
    float b[MS];
    const uint32_t r0 = in_ptr[v], r1 = in_ptr[v + 1];
    if (r1 > r0) {
#pragma unroll
        for (int i = 0; i < MS; ++i) b[i] = (UNI || i < S) ? 1.0f : 0.0f;
        for (uint32_t p = r0; p < r1; ++p) {
            float mm[MS];
            ldv<MS>(msg + (size_t)p * MS, mm);
            combine<MS, UNI>(b, mm, S);
        }
    } else {
        ldv<MS>(belief + (size_t)v * MS, b);
    }
    normalise<MS, UNI>(b, S);
    stv<MS>(belief + (size_t)v * MS, b);
}

void tree_clear(bp_graph *g) {
    TreeData &t = g->tree;
    if (t.exec) cudaGraphExecDestroy(t.exec);
    void *sched[] = {t.q_joint, t.q_joff, t.q_lvidx, t.q_y, t.q_pos, t.q_dst, t.s_in, t.s_out, t.s_lidx, t.s_S};
    for (void *p : sched)
        if (p) cudaFree(p);
    if (t.d_wave_off) cudaFree(t.d_wave_off);
    if (t.d_bar) cudaFree(t.d_bar);
    if (t.d_node_level) cudaFree(t.d_node_level);
    if (t.d_node_lidx) cudaFree(t.d_node_lidx);
    if (t.d_wave_nodes) cudaFree(t.d_wave_nodes);
    free(t.levels_host);
    free(t.wave_off);
    free(t.level_wave_begin);
    t = TreeData();
}

// waves of caller-given (or host-built) level lists, split on the host
int tree_prepare_host(bp_graph *g, const uint32_t *levels, uint32_t num_levels) {
    const uint32_t V = g->V;
    if (g->new_to_old) return set_error(BP_ERR_STATE, "tree BP on a renumbered graph (BP_GRAPH_REORDER_BY_OUT_DEGREE)");
    TreeData &t = g->tree;
    if (t.ready && t.num_levels == num_levels &&
        (V == 0 || (t.levels_host && memcmp(t.levels_host, levels, sizeof(uint32_t) * 2 * (size_t)V) == 0)))
        return BP_OK;
    tree_clear(g);
    if (num_levels == 0) return set_error(BP_ERR_STATE, "no levels (call init_levels_to_nodes first)");
    int st;
    if ((st = ensure_out_csr(g))) return st;
    if ((st = ensure_host_in_ptr(g))) return st;
    std::vector<uint32_t> in_src(g->E ? g->E : 1);
    if (g->E) BP_CUDA(cudaMemcpy(in_src.data(), g->in_src, sizeof(uint32_t) * g->E, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> node_level(V ? V : 1), node_lidx(V ? V : 1), wave_nodes(V ? V : 1);
    t.level_wave_begin = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)num_levels + 1));
    t.levels_host = (uint32_t *)malloc(sizeof(uint32_t) * (2 * (size_t)V + 1));
    if (V) memcpy(t.levels_host, levels, sizeof(uint32_t) * 2 * (size_t)V);
    uint32_t total = 0;
    int rc = bp_tree_waves(V, levels, num_levels, g->in_ptr_host, in_src.data(), node_level.data(),
                           node_lidx.data(), wave_nodes.data(), &t.wave_off, t.level_wave_begin, &total);
    if (rc != 0) {
        tree_clear(g);
        return set_error(rc == -2 ? BP_ERR_NOMEM : BP_ERR_INVALID, "malformed level lists");
    }
    for (uint32_t v = 0; v < V; ++v)
        if (node_level[v] == 0xffffffffu) {
            tree_clear(g);
            return set_error(BP_ERR_GRAPH, "node %u is in no level", v);
        }
    t.total_waves = total;
    t.num_levels = num_levels;
    const size_t bytes = sizeof(uint32_t) * (V ? V : 1);
    BP_CUDA(cudaMalloc((void **)&t.d_node_level, bytes));
    BP_CUDA(cudaMalloc((void **)&t.d_node_lidx, bytes));
    BP_CUDA(cudaMalloc((void **)&t.d_wave_nodes, bytes));
    BP_CUDA(cudaMemcpy(t.d_node_level, node_level.data(), bytes, cudaMemcpyHostToDevice));
    BP_CUDA(cudaMemcpy(t.d_node_lidx, node_lidx.data(), bytes, cudaMemcpyHostToDevice));
    BP_CUDA(cudaMemcpy(t.d_wave_nodes, wave_nodes.data(), bytes, cudaMemcpyHostToDevice));
    t.ready = true;
    return BP_OK;
}

static int exclusive_scan(const uint32_t *in, uint32_t *out, int64_t n, cudaStream_t st) {
    size_t temp = 0;
    BP_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, temp, in, out, n, st));
    void *tmp = nullptr;
    BP_CUDA(cudaMallocAsync(&tmp, temp, st));
    cudaError_t e = cub::DeviceScan::ExclusiveSum(tmp, temp, in, out, n, st);
    cudaFreeAsync(tmp, st);
    if (e != cudaSuccess) return cuda_fail(e, "DeviceScan::ExclusiveSum", __FILE__, __LINE__);
    return BP_OK;
}

// the schedule-order arrays for the current levels (built once per level
// lists, before any capture)
template <int MS, bool UNI>
static int tree_q_build(bp_graph *g) {
    TreeData &t = g->tree;
    if (t.q_joint) return BP_OK;
    const uint32_t V = g->V, E = g->E;
    int st;
    if ((st = ensure_out_csr(g))) return st;
    const size_t ne = E ? E : 1, nv = V ? V : 1;
    BP_CUDA(cudaMalloc((void **)&t.s_in, sizeof(uint2) * nv));
    BP_CUDA(cudaMalloc((void **)&t.s_out, sizeof(uint32_t) * (nv + 1)));
    BP_CUDA(cudaMalloc((void **)&t.s_lidx, sizeof(uint32_t) * nv));
    BP_CUDA(cudaMalloc((void **)&t.s_S, nv));
    BP_CUDA(cudaMalloc((void **)&t.q_y, ne));
    BP_CUDA(cudaMalloc((void **)&t.q_joff, sizeof(uint32_t) * (ne + 1)));
    BP_CUDA(cudaMalloc((void **)&t.q_lvidx, sizeof(uint2) * ne));
    BP_CUDA(cudaMalloc((void **)&t.q_pos, sizeof(uint32_t) * ne));
    BP_CUDA(cudaMalloc((void **)&t.q_dst, sizeof(uint32_t) * ne));
    uint32_t *cnt = nullptr;
    BP_CUDA(cudaMallocAsync((void **)&cnt, sizeof(uint32_t) * (std::max(nv, ne) + 1), g->stream));
    BP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * (std::max(nv, ne) + 1), g->stream));
    if (V)
        k_ts_nodes<<<grid_for(V, 256), 256, 0, g->stream>>>(V, t.d_wave_nodes, g->in_ptr, g->out_ptr, t.d_node_lidx,
                                                            g->node_s, t.s_in, t.s_lidx, t.s_S, cnt);
    BP_CUDA(cudaGetLastError());
    if ((st = exclusive_scan(cnt, t.s_out, (int64_t)V + 1, g->stream))) return st;
    BP_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t) * (ne + 1), g->stream));
    if (V)
        k_tq_sizes<<<grid_for(V, 256), 256, 0, g->stream>>>(V, t.d_wave_nodes, t.s_out, g->out_ptr, g->out_dst,
                                                            g->node_s, t.q_y, cnt);
    BP_CUDA(cudaGetLastError());
    if ((st = exclusive_scan(cnt, t.q_joff, (int64_t)E + 1, g->stream))) return st;
    uint32_t total = 0;
    BP_CUDA(cudaMemcpyAsync(&total, t.q_joff + E, sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
    BP_CUDA(cudaStreamSynchronize(g->stream));
    cudaFreeAsync(cnt, g->stream);
    BP_CUDA(cudaMalloc((void **)&t.q_joint, sizeof(float) * ((size_t)total + 4)));
    BP_CUDA(cudaMalloc((void **)&t.d_wave_off, sizeof(uint32_t) * ((size_t)t.total_waves + 1)));
    BP_CUDA(cudaMemcpy(t.d_wave_off, t.wave_off, sizeof(uint32_t) * ((size_t)t.total_waves + 1),
                       cudaMemcpyHostToDevice));
    BP_CUDA(cudaMalloc((void **)&t.d_bar, 4 * sizeof(uint32_t)));
    BP_CUDA(cudaMemset(t.d_bar, 0, 4 * sizeof(uint32_t)));
    if (V)
        k_tq_fill<MS><<<grid_for(V, 256), 256, 0, g->stream>>>(V, t.d_wave_nodes, t.s_out, g->out_ptr, g->out_pos,
                                                               g->out_dst, g->node_s, t.q_y, t.q_joff, g->joint,
                                                               t.d_node_level, t.d_node_lidx, t.q_joint, t.q_lvidx,
                                                               t.q_pos, t.q_dst);
    BP_CUDA(cudaGetLastError());
    BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

static TreeArgs tree_args(bp_graph *g) {
    TreeData &t = g->tree;
    TreeArgs a;
    a.nodes = t.d_wave_nodes;
    a.s_in = t.s_in;
    a.s_out = t.s_out;
    a.s_lidx = t.s_lidx;
    a.s_S = t.s_S;
    a.q_pos = t.q_pos;
    a.q_dst = t.q_dst;
    a.q_lvidx = t.q_lvidx;
    a.q_y = t.q_y;
    a.q_joff = t.q_joff;
    a.q_joint = t.q_joint;
    a.belief = g->belief;
    a.msg = g->msg[0];
    a.visited = g->visited;
    return a;
}

// mark: set the level-0 visited flags (graph.h calls; bp_tree derives them)
template <int MS, bool UNI>
static int launch_start(bp_graph *g, int mark) {
    TreeData &t = g->tree;
    const uint32_t w0 = t.level_wave_begin[0], w1 = t.level_wave_begin[1];
    if (w1 == w0) return BP_OK;
    const uint32_t lo = t.wave_off[w0], n = t.wave_off[w1] - lo;
    k_tree_start<MS, UNI><<<grid_for(n, 128), 128, 0, g->stream>>>(tree_args(g), lo, n, mark);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

// lanes per node of a wave: the widest group (1, 2, 4, 8, 16 or 32 lanes)
// that keeps the wave within three residencies of the GPU (148 SMs x 2048
// threads x 3), so small waves spread each node's chain of dependent loads
// over a group and big ones keep a thread per node (on a 2M-node random tree
// budgets from 0.6M to 0.96M threads were equally fast, 2.56M lost 23 %);
// BP_TREE_GROUP_THREADS overrides the budget (sweeps)
constexpr uint64_t kGroupWaveThreads = 148ull * 2048ull * 3ull;
static uint64_t group_wave_threads() {
    static uint64_t t = 0;
    if (!t) {
        const char *env = getenv("BP_TREE_GROUP_THREADS");
        t = env ? (uint64_t)atoll(env) : kGroupWaveThreads;
        if (!t) t = 1;
    }
    return t;
}
static int wave_group(uint64_t n) {
    const uint64_t t = group_wave_threads();
    for (int gsz = 32; gsz >= 2; gsz >>= 1)
        if (n * gsz <= t) return gsz;
    return 1;
}

// wave kernels may start while the kernel ahead drains (programmatic
// dependent launch): they read the schedule first and wait before the
// messages; BP_TREE_PDL=0 launches them one after another
static bool tree_pdl() {
    static int on = -1;
    if (on < 0) {
        const char *env = getenv("BP_TREE_PDL");
        on = (env && env[0] == '0') ? 0 : 1;
    }
    return on != 0;
}

template <typename... KArgs, typename... Args>
static cudaError_t launch_wave(void (*kern)(KArgs...), unsigned grid, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(128);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = tree_pdl() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <int MS, bool UNI, int G>
static cudaError_t launch_wave_group(bp_graph *g, uint32_t k0, uint32_t n, uint32_t level, int mode) {
    return launch_wave(k_tree_wave_group<MS, UNI, G>, grid_for((uint64_t)n * G, 128), g->stream, tree_args(g), k0, n,
                       level, mode);
}

// BP_TREE_TAIL=1 runs each run of warp-per-node waves as one cooperative
// launch (read when the launch sequence is built).  Off by default: on the
// 2M-node random tree it measured 0.98 ms per tree against 0.86 ms with one
// programmatic-dependent launch per wave -- the grid barrier over every
// co-resident block costs more than the launch it saves.
static bool tree_tail_on() {
    const char *env = getenv("BP_TREE_TAIL");
    return env && env[0] == '1';
}

// waves [wa, wb) of `level` (every one a warp per node) as one cooperative
// launch of k_tree_tail
template <int MS, bool UNI>
static int launch_tail(bp_graph *g, uint32_t level, uint32_t wa, uint32_t wb, int mode) {
    TreeData &t = g->tree;
    static int bps = 0;
    if (!bps) BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_tree_tail<MS, UNI>, 256, 0));
    int dev = 0, sms = 0;
    BP_CUDA(cudaGetDevice(&dev));
    BP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    uint32_t nmax = 0;
    for (uint32_t w = wa; w < wb; ++w) nmax = std::max(nmax, t.wave_off[w + 1] - t.wave_off[w]);
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)bps * sms,
                                                                           ((uint64_t)nmax * 32 + 255) / 256));
    TreeTailArgs a;
    a.t = tree_args(g);
    a.wave_off = t.d_wave_off;
    a.w0 = wa;
    a.w1 = wb;
    a.level = level;
    a.mode = mode;
    a.bar = t.d_bar;
    // arrivals and generation restart at zero; a failure flag set by an
    // earlier launch stays set for bp_tree to report
    BP_CUDA(cudaMemsetAsync(t.d_bar, 0, 2 * sizeof(uint32_t), g->stream));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(256);
    cfg.stream = g->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    BP_CUDA(cudaLaunchKernelEx(&cfg, k_tree_tail<MS, UNI>, a));
    return BP_OK;
}

// the waves of `level`; mode 0 (graph.h calls) reads and then sets the
// visited flags, modes 1 and 2 (bp_tree's upward and downward passes) derive
// them from the levels
template <int MS, bool UNI>
static int launch_level(bp_graph *g, uint32_t level, int mode) {
    TreeData &t = g->tree;
    const uint32_t w0 = t.level_wave_begin[level], w1 = t.level_wave_begin[level + 1];
    for (uint32_t w = w0; w < w1; ++w) {
        const uint32_t lo = t.wave_off[w], n = t.wave_off[w + 1] - lo;
        if (!n) continue;
        if (tree_tail_on() && wave_group(n) == 32) {
            // the run of warp-per-node waves that starts here
            uint32_t we = w + 1;
            while (we < w1 && wave_group(t.wave_off[we + 1] - t.wave_off[we]) == 32) ++we;
            if (we - w >= 2) {
                int st = launch_tail<MS, UNI>(g, level, w, we, mode);
                if (st) return st;
                w = we - 1;
                continue;
            }
        }
        cudaError_t le;
        switch (wave_group(n)) {
        case 32: le = launch_wave_group<MS, UNI, 32>(g, lo, n, level, mode); break;
        case 16: le = launch_wave_group<MS, UNI, 16>(g, lo, n, level, mode); break;
        case 8: le = launch_wave_group<MS, UNI, 8>(g, lo, n, level, mode); break;
        case 4: le = launch_wave_group<MS, UNI, 4>(g, lo, n, level, mode); break;
        case 2: le = launch_wave_group<MS, UNI, 2>(g, lo, n, level, mode); break;
        default: le = launch_wave(k_tree_wave<MS, UNI>, grid_for(n, 128), g->stream, tree_args(g), lo, n, level, mode);
        }
        if (le != cudaSuccess) return cuda_fail(le, "cudaLaunchKernelEx", __FILE__, __LINE__);
        BP_CUDA(cudaGetLastError());
    }
    if (w1 > w0 && mode == 0) {
        const uint32_t lo = t.wave_off[w0], n = t.wave_off[w1] - lo;
        k_mark_visited<<<grid_for(n, 256), 256, 0, g->stream>>>(t.d_wave_nodes + lo, n, g->visited);
        BP_CUDA(cudaGetLastError());
    }
    return BP_OK;
}

template <int MS, bool UNI>
static int launch_marginalize(bp_graph *g) {
    if (g->V == 0) return BP_OK;
    k_tree_marginalize<MS, UNI><<<grid_for(g->V, 256), 256, 0, g->stream>>>(g->V, g->in_ptr, g->node_s, g->msg[0],
                                                                             g->belief);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

static int dispatch_q_build(bp_graph *g) { BP_DISPATCH_MS(g->ms, g->uniform != 0, tree_q_build, g); }
static int dispatch_start(bp_graph *g, int mark) { BP_DISPATCH_MS(g->ms, g->uniform != 0, launch_start, g, mark); }
static int dispatch_level(bp_graph *g, uint32_t l, int mode) {
    BP_DISPATCH_MS(g->ms, g->uniform != 0, launch_level, g, l, mode);
}
static int dispatch_marginalize(bp_graph *g) { BP_DISPATCH_MS(g->ms, g->uniform != 0, launch_marginalize, g); }

}  // namespace bpx

using namespace bpx;

extern "C" {

int bp_tree_build_levels(bp_graph *g, uint32_t *levels, uint32_t *num_levels) {
    if (!g || !num_levels) return set_error(BP_ERR_INVALID, "null argument");
    if (g->new_to_old) return set_error(BP_ERR_STATE, "tree BP on a renumbered graph (BP_GRAPH_REORDER_BY_OUT_DEGREE)");
    int st;
    // the device build; BP_TREE_LEVELS=host, or a caller's non-zero level
    // count to continue from (the reference never resets num_levels), takes
    // the host build
    const char *env = getenv("BP_TREE_LEVELS");
    if (*num_levels == 0 && !(env && env[0] == 'h')) return tree_build_levels_gpu(g, levels, num_levels);
    if ((st = ensure_out_csr(g))) return st;
    if ((st = ensure_host_in_ptr(g))) return st;
    const uint32_t V = g->V, E = g->E;
    std::vector<uint32_t> out_ptr((size_t)V + 1), out_dst(E ? E : 1);
    BP_CUDA(cudaMemcpy(out_ptr.data(), g->out_ptr, sizeof(uint32_t) * ((size_t)V + 1), cudaMemcpyDeviceToHost));
    if (E) BP_CUDA(cudaMemcpy(out_dst.data(), g->out_dst, sizeof(uint32_t) * E, cudaMemcpyDeviceToHost));
    std::vector<uint32_t> lv(2 * (size_t)V + 1, 0);
    uint32_t nl = *num_levels;
    int rc = bp_levels_from_csr(V, g->in_ptr_host, out_ptr.data(), out_dst.data(), lv.data(), &nl);
    if (rc == -2) return set_error(BP_ERR_NOMEM, "host allocation failed");
    if (rc == -1) return set_error(BP_ERR_GRAPH, "a node is unreachable from the in-degree<=2 seed set");
    *num_levels = nl;
    if (levels) memcpy(levels, lv.data(), sizeof(uint32_t) * 2 * (size_t)V);
    return tree_prepare_host(g, lv.data(), nl);
}

int bp_tree_set_levels(bp_graph *g, const uint32_t *levels, uint32_t num_levels) {
    if (!g || (!levels && g->V)) return set_error(BP_ERR_INVALID, "null argument");
    return tree_prepare_host(g, levels, num_levels);
}

int bp_tree_start(bp_graph *g) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    if (!g->tree.ready) return set_error(BP_ERR_STATE, "tree levels not set");
    int st = dispatch_q_build(g);
    return st ? st : dispatch_start(g, 1);
}

int bp_tree_level(bp_graph *g, uint32_t level) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    if (!g->tree.ready) return set_error(BP_ERR_STATE, "tree levels not set");
    if (level >= g->tree.num_levels) return set_error(BP_ERR_INVALID, "level %u >= num_levels %u", level,
                                                      g->tree.num_levels);
    int st = dispatch_q_build(g);
    return st ? st : dispatch_level(g, level, 0);
}

int bp_tree_reset_visited(bp_graph *g) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    if (g->V) BP_CUDA(cudaMemsetAsync(g->visited, 0, g->V, g->stream));
    return BP_OK;
}

int bp_tree_marginalize(bp_graph *g) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    return dispatch_marginalize(g);
}

// the whole schedule of c_benchmark/main.c:224-236 on the graph's stream:
// reset_visited, start, levels 1 .. L-2, reset_visited, levels L-1 .. 1,
// marginalize.  The visited flags of each step follow from the levels
// (modes 1 and 2 of launch_level); the flags the schedule leaves are written
// at the end.
static int tree_enqueue(bp_graph *g) {
    int st;
    const uint32_t L = g->tree.num_levels;
    if ((st = dispatch_start(g, 0))) return st;
    for (uint32_t l = 1; l + 1 < L; ++l)
        if ((st = dispatch_level(g, l, 1))) return st;
    for (uint32_t l = L - 1; l > 0; --l)
        if ((st = dispatch_level(g, l, 2))) return st;
    if ((st = dispatch_marginalize(g))) return st;
    if (g->V) {
        k_final_visited<<<grid_for(g->V, 256), 256, 0, g->stream>>>(g->V, g->tree.d_node_level, g->visited);
        BP_CUDA(cudaGetLastError());
    }
    return BP_OK;
}

int bp_tree(bp_graph *g, bp_tree_result *res) {
    NvtxRange nvtx("bp_tree");
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    int st;
    if (!g->tree.ready) {
        uint32_t nl = 0;
        if ((st = bp_tree_build_levels(g, nullptr, &nl))) return st;
    }
    if ((st = dispatch_q_build(g))) return st;
    TreeData &t = g->tree;
    const uint32_t L = t.num_levels;
    uint32_t waves = t.level_wave_begin[1] - t.level_wave_begin[0] ? 1 : 0;
    for (uint32_t l = 1; l + 1 < L; ++l) waves += t.level_wave_begin[l + 1] - t.level_wave_begin[l];
    for (uint32_t l = L - 1; l > 0; --l) waves += t.level_wave_begin[l + 1] - t.level_wave_begin[l];
    // one launch per wave: the sequence is fixed for the levels, so it is
    // captured once into a CUDA graph and replayed
    if (!t.exec) {
        cudaGraph_t graph = nullptr;
        BP_CUDA(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
        st = tree_enqueue(g);
        cudaError_t ce = cudaStreamEndCapture(g->stream, &graph);
        if (st) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
        cudaError_t ie = cudaGraphInstantiate(&t.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            t.exec = nullptr;
            return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
        }
    }
    BP_CUDA(cudaEventRecord(g->ev0, g->stream));
    BP_CUDA(cudaGraphLaunch(t.exec, g->stream));
    BP_CUDA(cudaEventRecord(g->ev1, g->stream));
    BP_CUDA(cudaStreamSynchronize(g->stream));
    if (t.d_bar) {
        uint32_t fail = 0;
        BP_CUDA(cudaMemcpy(&fail, t.d_bar + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost));
        if (fail) {
            BP_CUDA(cudaMemset(t.d_bar + 2, 0, sizeof(uint32_t)));
            return set_error(BP_ERR_TIMEOUT, "a bounded grid-barrier wait of the tree's small waves timed out");
        }
    }
    if (res) {
        res->num_levels = L;
        res->num_waves = waves;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, g->ev0, g->ev1);
        res->elapsed_ms = ms;
    }
    return BP_OK;
}

}  // extern "C"
