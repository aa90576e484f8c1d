// levels_gpu.cu -- the tree schedule's level lists and waves, built on the device.
//
// Level lists (init_levels_to_nodes, graph.c:806-827): level 0 lists, in
// ascending id, the nodes with in-degree <= 2 (fill_in_leaf_nodes_in_index,
// graph.c:753-772); each later level lists the out-neighbours of the previous
// level that are not listed yet, in the order the reference's visit_node
// (graph.c:774-804) appends them: by the position of the first previous-level
// node that reaches them, then by that node's out-edge order.  Here one BFS
// round per level: every out-edge of the frontier into an unlisted node offers
// the key (frontier position, out-edge rank) with a 64-bit atomicMin, the
// first offer also appends the node to a candidate list, and a radix sort of
// the candidates by their final (smallest) key gives the reference's order.
// O(V + E) work plus one sort per level, instead of the reference's O(V^2)
// list scan.
//
// Waves (the same split as levels.c's bp_tree_waves): node k of a level runs
// one wave after the latest earlier node of its level with an edge into it.
// wave(u) = 1 + max wave(s) over such in-neighbours s is a longest path in the
// level's DAG (edges go from lower to higher list position), found by
// monotone relaxation rounds over all nodes; a stable radix sort by
// (level, wave) then lays the waves out contiguously in list order.  A level
// whose chains are longer than kMaxWaveRounds is handed to the host split.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_select.cuh>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "bp_device.cuh"
#include "bp_internal.h"
#include "bp_levels.h"

namespace bpx {

constexpr uint64_t kNoKey = ~0ull;
constexpr uint32_t kMaxWaveRounds = 256;

__global__ void k_leaf_flags(uint32_t V, const uint32_t *__restrict__ in_ptr, uint8_t *__restrict__ listed,
                             uint32_t *__restrict__ iota) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    listed[v] = (in_ptr[v + 1] - in_ptr[v] <= 2) ? 1 : 0;
    iota[v] = v;
}

__global__ void k_fill_u64(unsigned long long *__restrict__ a, uint32_t n, unsigned long long x) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = x;
}

// every out-edge of the frontier into an unlisted node offers (position, rank)
__global__ void k_level_discover(const uint32_t *__restrict__ front, uint32_t n, const uint32_t *__restrict__ out_ptr,
                                 const uint32_t *__restrict__ out_dst, const uint8_t *__restrict__ listed,
                                 unsigned long long *__restrict__ key, uint32_t *__restrict__ cand,
                                 uint32_t *__restrict__ ncand) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t u = front[i], q0 = out_ptr[u], q1 = out_ptr[u + 1];
    for (uint32_t q = q0; q < q1; ++q) {
        const uint32_t d = out_dst[q];
        if (listed[d]) continue;
        const unsigned long long k = ((unsigned long long)i << 32) | (q - q0);
        if (atomicMin(key + d, k) == kNoKey) cand[atomicAdd(ncand, 1u)] = d;
    }
}

// the candidates' final keys; their key slots reset and the nodes listed
__global__ void k_level_take(const uint32_t *__restrict__ cand, uint32_t n, unsigned long long *__restrict__ key,
                             uint8_t *__restrict__ listed, unsigned long long *__restrict__ keys_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t d = cand[i];
    keys_out[i] = key[d];
    key[d] = kNoKey;
    listed[d] = 1;
}

__global__ void k_level_assign(const uint32_t *__restrict__ nodes, uint32_t n, uint32_t level,
                               uint32_t *__restrict__ node_level, uint32_t *__restrict__ node_lidx) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    node_level[nodes[i]] = level;
    node_lidx[nodes[i]] = i;
}

__global__ void k_wave_round(uint32_t V, const uint32_t *__restrict__ in_ptr, const uint32_t *__restrict__ in_src,
                             const uint32_t *__restrict__ node_level, const uint32_t *__restrict__ node_lidx,
                             uint32_t *wave, uint32_t *__restrict__ changed) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= V) return;
    const uint32_t l = node_level[u], k = node_lidx[u];
    uint32_t w = 0;
    for (uint32_t p = in_ptr[u]; p < in_ptr[u + 1]; ++p) {
        const uint32_t s = in_src[p];
        if (node_level[s] == l && node_lidx[s] < k) w = max(w, ((volatile uint32_t *)wave)[s] + 1u);
    }
    if (w > wave[u]) {
        wave[u] = w;
        *changed = 1u;
    }
}

__global__ void k_wave_keys(const uint32_t *__restrict__ nodes, uint32_t V, const uint32_t *__restrict__ node_level,
                            const uint32_t *__restrict__ wave, unsigned long long *__restrict__ keys) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= V) return;
    const uint32_t u = nodes[k];
    keys[k] = ((unsigned long long)node_level[u] << 32) | wave[u];
}

__global__ void k_run_heads(const unsigned long long *__restrict__ keys, uint32_t V, uint8_t *__restrict__ head,
                            uint32_t *__restrict__ iota) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= V) return;
    head[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1 : 0;
    iota[k] = k;
}

__global__ void k_run_levels(const unsigned long long *__restrict__ keys, const uint32_t *__restrict__ starts,
                             uint32_t n, uint32_t *__restrict__ level) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) level[i] = (uint32_t)(keys[starts[i]] >> 32);
}

static int bits_for(uint64_t x) {
    int b = 1;
    while (b < 64 && (x >> b)) ++b;
    return b;
}

// scoped device buffers from the stream-ordered pool
struct PoolBufs {
    cudaStream_t s;
    std::vector<void *> p;
    explicit PoolBufs(cudaStream_t s_) : s(s_) {}
    ~PoolBufs() {
        for (void *x : p) cudaFreeAsync(x, s);
    }
    template <class T>
    cudaError_t get(T **out, size_t n) {
        void *x = nullptr;
        cudaError_t e = cudaMallocAsync(&x, sizeof(T) * (n ? n : 1), s);
        if (e == cudaSuccess) p.push_back(x);
        *out = (T *)x;
        return e;
    }
};

int tree_build_levels_gpu(bp_graph *g, uint32_t *levels_out, uint32_t *num_levels_out) {
    const uint32_t V = g->V;
    cudaStream_t st = g->stream;
    int rc;
    StageTrace trace(st, "levels");
    if ((rc = ensure_out_csr(g))) return rc;
    trace.mark("source-sorted csr");
    tree_clear(g);
    TreeData &t = g->tree;
    PoolBufs pb(st);
    uint8_t *listed = nullptr, *head = nullptr;
    uint32_t *iota = nullptr, *lv = nullptr, *cand = nullptr, *counter = nullptr, *wave = nullptr,
             *sorted_nodes = nullptr, *starts = nullptr, *run_level = nullptr;
    unsigned long long *key = nullptr, *ckeys = nullptr, *ckeys_sorted = nullptr;
    BP_CUDA(pb.get(&listed, V));
    BP_CUDA(pb.get(&head, V));
    BP_CUDA(pb.get(&iota, V));
    BP_CUDA(pb.get(&lv, V));
    BP_CUDA(pb.get(&cand, V));
    BP_CUDA(pb.get(&counter, 2));
    BP_CUDA(pb.get(&wave, V));
    BP_CUDA(pb.get(&starts, V));
    BP_CUDA(pb.get(&run_level, V));
    BP_CUDA(pb.get(&key, V));
    BP_CUDA(pb.get(&ckeys, V));
    BP_CUDA(pb.get(&ckeys_sorted, V));
    const size_t bytes = sizeof(uint32_t) * (V ? V : 1);
    BP_CUDA(cudaMalloc((void **)&t.d_node_level, bytes));
    BP_CUDA(cudaMalloc((void **)&t.d_node_lidx, bytes));
    BP_CUDA(cudaMalloc((void **)&t.d_wave_nodes, bytes));
    sorted_nodes = t.d_wave_nodes;
    uint32_t hc = 0;
    uint32_t *h_count = &hc;

    trace.mark("buffers");
    // ---- level 0: ascending ids with in-degree <= 2
    const unsigned gv = grid_for(V, 256);
    k_leaf_flags<<<gv, 256, 0, st>>>(V, g->in_ptr, listed, iota);
    k_fill_u64<<<gv, 256, 0, st>>>(key, V, kNoKey);
    BP_CUDA(cudaGetLastError());
    size_t tb = 0, tb2 = 0;
    BP_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, iota, listed, lv, counter, (int64_t)V, st));
    BP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb2, ckeys, ckeys_sorted, cand, lv, (int64_t)V, 0, 64, st));
    tb = std::max(tb, tb2);
    void *temp = nullptr;
    BP_CUDA(pb.get((unsigned char **)&temp, tb));
    BP_CUDA(cub::DeviceSelect::Flagged(temp, tb, iota, listed, lv, counter, (int64_t)V, st));
    BP_CUDA(cudaMemcpyAsync(h_count, counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    BP_CUDA(cudaStreamSynchronize(st));
    std::vector<uint32_t> off(1, 0);   // list positions where each level starts
    uint32_t end = *h_count;
    if (end) {
        k_level_assign<<<grid_for(end, 256), 256, 0, st>>>(lv, end, 0, t.d_node_level, t.d_node_lidx);
        BP_CUDA(cudaGetLastError());
    }

    // ---- BFS rounds
    uint32_t lo = 0;
    while (end < V) {
        const uint32_t n = end - lo;
        BP_CUDA(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st));
        if (n) {
            k_level_discover<<<grid_for(n, 128), 128, 0, st>>>(lv + lo, n, g->out_ptr, g->out_dst, listed, key, cand,
                                                               counter);
            BP_CUDA(cudaGetLastError());
        }
        BP_CUDA(cudaMemcpyAsync(h_count, counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        BP_CUDA(cudaStreamSynchronize(st));
        const uint32_t c = *h_count;
        if (c == 0) {
            tree_clear(g);
            return set_error(BP_ERR_GRAPH, "a node is unreachable from the in-degree<=2 seed set");
        }
        k_level_take<<<grid_for(c, 256), 256, 0, st>>>(cand, c, key, listed, ckeys);
        BP_CUDA(cudaGetLastError());
        BP_CUDA(cub::DeviceRadixSort::SortPairs(temp, tb, ckeys, ckeys_sorted, cand, lv + end, (int64_t)c, 0,
                                                32 + bits_for(n), st));
        off.push_back(end);
        k_level_assign<<<grid_for(c, 256), 256, 0, st>>>(lv + end, c, (uint32_t)(off.size() - 1), t.d_node_level,
                                                         t.d_node_lidx);
        BP_CUDA(cudaGetLastError());
        lo = end;
        end += c;
    }
    const uint32_t L = (uint32_t)off.size();
    trace.mark("level lists");

    // ---- waves: relaxation rounds to the longest-path fixed point
    bool converged = V == 0;
    if (V) {
        BP_CUDA(cudaMemsetAsync(wave, 0, bytes, st));
        for (uint32_t r = 0; r < kMaxWaveRounds; ++r) {
            BP_CUDA(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st));
            k_wave_round<<<gv, 256, 0, st>>>(V, g->in_ptr, g->in_src, t.d_node_level, t.d_node_lidx, wave, counter);
            BP_CUDA(cudaGetLastError());
            BP_CUDA(cudaMemcpyAsync(h_count, counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
            BP_CUDA(cudaStreamSynchronize(st));
            if (*h_count == 0) {
                converged = true;
                break;
            }
        }
    }

    trace.mark("wave rounds");
    // the reference's levels_to_nodes layout: offsets, then the list at [V, 2V)
    std::vector<uint32_t> host_levels;
    const bool want_host = levels_out != nullptr || !converged;
    if (want_host) {
        host_levels.assign(2 * (size_t)V + 1, 0);
        for (uint32_t l = 0; l < L; ++l) host_levels[l] = V + off[l];
        if (V) BP_CUDA(cudaMemcpyAsync(host_levels.data() + V, lv, bytes, cudaMemcpyDeviceToHost, st));
        BP_CUDA(cudaStreamSynchronize(st));
        if (levels_out) memcpy(levels_out, host_levels.data(), sizeof(uint32_t) * 2 * (size_t)V);
    }
    trace.mark("list to host");
    *num_levels_out = L;
    if (!converged) {
        // chains longer than the round cap: the host split on the same list
        tree_clear(g);
        return tree_prepare_host(g, host_levels.data(), L);
    }

    // ---- stable sort of the list by (level, wave); one run per wave
    uint32_t nruns = 0;
    std::vector<uint32_t> run_start, run_lvl;
    if (V) {
        k_wave_keys<<<gv, 256, 0, st>>>(lv, V, t.d_node_level, wave, ckeys);
        BP_CUDA(cudaGetLastError());
        BP_CUDA(cub::DeviceRadixSort::SortPairs(temp, tb, ckeys, ckeys_sorted, lv, sorted_nodes, (int64_t)V, 0,
                                                32 + bits_for(L), st));
        k_run_heads<<<gv, 256, 0, st>>>(ckeys_sorted, V, head, iota);
        BP_CUDA(cudaGetLastError());
        BP_CUDA(cub::DeviceSelect::Flagged(temp, tb, iota, head, starts, counter, (int64_t)V, st));
        BP_CUDA(cudaMemcpyAsync(h_count, counter, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        BP_CUDA(cudaStreamSynchronize(st));
        nruns = *h_count;
        k_run_levels<<<grid_for(nruns, 256), 256, 0, st>>>(ckeys_sorted, starts, nruns, run_level);
        BP_CUDA(cudaGetLastError());
        run_start.resize(nruns);
        run_lvl.resize(nruns);
        BP_CUDA(cudaMemcpyAsync(run_start.data(), starts, sizeof(uint32_t) * nruns, cudaMemcpyDeviceToHost, st));
        BP_CUDA(cudaMemcpyAsync(run_lvl.data(), run_level, sizeof(uint32_t) * nruns, cudaMemcpyDeviceToHost, st));
        BP_CUDA(cudaStreamSynchronize(st));
    }
    trace.mark("wave layout");
    t.wave_off = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)nruns + 1));
    t.level_wave_begin = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)L + 1));
    if (!t.wave_off || !t.level_wave_begin) {
        tree_clear(g);
        return set_error(BP_ERR_NOMEM, "host allocation failed");
    }
    for (uint32_t w = 0; w < nruns; ++w) t.wave_off[w] = run_start[w];
    t.wave_off[nruns] = V;
    uint32_t w = 0;
    for (uint32_t l = 0; l <= L; ++l) {
        while (w < nruns && run_lvl[w] < l) ++w;
        t.level_wave_begin[l] = w;
    }
    t.total_waves = nruns;
    t.num_levels = L;
    if (want_host) {
        t.levels_host = (uint32_t *)malloc(sizeof(uint32_t) * (2 * (size_t)V + 1));
        if (t.levels_host) memcpy(t.levels_host, host_levels.data(), sizeof(uint32_t) * 2 * (size_t)V);
    }
    t.ready = true;
    return BP_OK;
}

}  // namespace bpx
