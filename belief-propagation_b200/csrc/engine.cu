// engine.cu -- device graph construction, state transfer, error plumbing.
//
// bp_graph_create turns an edge list in insertion order into the
// destination-sorted layout described in bp_internal.h.  The sort is a
// stable LSD radix sort by destination, so within a node the in-edges keep
// insertion order -- exactly the order of the reference's dest-CSR
// (graph.c:285-313) -- unless the caller passes that CSR explicitly.
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <chrono>
#include <vector>

#include "bp_device.cuh"
#include "bp_internal.h"

namespace bpx {

static thread_local char g_last_error[512] = "";

int set_error(int status, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return status;
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    int st = (e == cudaErrorMemoryAllocation) ? BP_ERR_NOMEM
           : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? BP_ERR_NO_DEVICE
           : BP_ERR_CUDA;
    return set_error(st, "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file, line);
}

// Graph buffers come from the device's stream-ordered memory pool, whose
// release threshold is raised once per device: memory freed by one graph
// stays cached for the next instead of going back to the driver, so
// creating and destroying graphs of similar size costs no cudaMalloc /
// cudaFree round trips.  bp_release_cached_memory() trims the pool.
static std::mutex g_pool_mutex;
static bool g_pool_ready[64];

static void ensure_pool(int dev) {
    if (dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (g_pool_ready[dev]) return;

    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t threshold = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold);
    }
    g_pool_ready[dev] = true;
}

int dev_alloc(bp_graph *g, void **p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocAsync(p, bytes, g->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_fail(e, "cudaMallocAsync", __FILE__, __LINE__);
    }
    g->device_bytes += bytes;
    return BP_OK;
}

// the pinned control blocks of loopy runs, reused across graphs
static std::mutex g_pinned_mutex;
static std::vector<LoopyCtl *> g_pinned_free;

static LoopyCtl *pinned_ctl() {
    {
        std::lock_guard<std::mutex> lock(g_pinned_mutex);
        if (!g_pinned_free.empty()) {
            LoopyCtl *c = g_pinned_free.back();
            g_pinned_free.pop_back();
            return c;
        }
    }
    LoopyCtl *c = nullptr;
    if (cudaMallocHost((void **)&c, sizeof(LoopyCtl)) != cudaSuccess) return nullptr;
    return c;
}

static void release_pinned_ctl(LoopyCtl *c) {
    if (!c) return;
    std::lock_guard<std::mutex> lock(g_pinned_mutex);
    g_pinned_free.push_back(c);
}

int ensure_staging(bp_graph *g, size_t bytes) {
    if (g->staging_bytes >= bytes) return BP_OK;
    if (g->staging) {
        cudaFreeAsync(g->staging, g->stream);
        g->device_bytes -= g->staging_bytes;
        g->staging = nullptr;
        g->staging_bytes = 0;
    }
    int st = dev_alloc(g, (void **)&g->staging, bytes);
    if (st == BP_OK) g->staging_bytes = bytes;
    return st;
}

// ---------------------------------------------------------------- kernels --

// row pointers from keys sorted ascending (ptr[v] = first position whose key
// >= v), in two streaming passes: the end of each key's run is written at
// end[key] (one write per key present; end is zeroed first), then ptr[v + 1]
// = max(end[0..v]) and ptr[0] = 0.  A kernel that wrote ptr[lo..hi] for the
// keys missing between two runs put long runs of absent keys (nodes without
// in-edges, grouped together by the renumbering) on single threads.
__global__ void k_run_ends(const uint32_t *__restrict__ keys, uint32_t E, uint32_t *__restrict__ end) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= E) return;
    const uint32_t k = keys[p];
    if (p + 1 == E || keys[p + 1] != k) end[k] = (uint32_t)(p + 1);
}

struct MaxU32 {
    __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const { return a > b ? a : b; }
};

// node_list (V entries, struct graph layout) -> ptr[V+1]
__global__ void k_ptr_from_node_list(const uint32_t *__restrict__ nl, uint32_t V, uint32_t E,
                                     uint32_t *__restrict__ ptr) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < V) ptr[v] = nl[v];
    if (v == V) ptr[V] = E;
}

// in_src (and pos_dims) at every position from the edge ids there: a
// gather by edge id (graphs given with the caller's destination CSR)
__global__ void k_positions(const uint32_t *__restrict__ pos_edge, const uint32_t *__restrict__ src,
                            const uint32_t *__restrict__ dst, uint32_t E,
                            const uint8_t *__restrict__ node_s, uint32_t *__restrict__ in_src,
                            uint8_t *__restrict__ pos_dims) {
    uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= E) return;
    uint32_t e = pos_edge[p];
    uint32_t s = src[e];
    in_src[p] = s;
    if (pos_dims) pos_dims[p] = (uint8_t)(node_s[s] | (node_s[dst[e]] << 4));
}

// the destination sort carries (source, edge id) as one 64-bit value, so
// in_src and pos_edge come out of the sort in position order without a
// gather by edge id (each such random 4-byte read cost about 128 B of DRAM)
__global__ void k_pack_src_id(const uint32_t *__restrict__ src, uint32_t E, uint64_t *__restrict__ out) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < E) out[e] = ((uint64_t)src[e] << 32) | e;
}

__global__ void k_unpack_positions(const uint64_t *__restrict__ vals, const uint32_t *__restrict__ dst_sorted,
                                   uint32_t E, const uint8_t *__restrict__ node_s, uint32_t *__restrict__ in_src,
                                   uint32_t *__restrict__ pos_edge, uint8_t *__restrict__ pos_dims) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= E) return;
    const uint64_t v = vals[p];
    const uint32_t s = (uint32_t)(v >> 32);
    in_src[p] = s;
    pos_edge[p] = (uint32_t)v;
    if (pos_dims) pos_dims[p] = (uint8_t)(node_s[s] | (node_s[dst_sorted[p]] << 4));
}

__global__ void k_states_u8(const uint32_t *__restrict__ s32, uint32_t V, uint32_t uniform,
                            uint8_t *__restrict__ s8) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v < V) s8[v] = (uint8_t)(s32 ? s32[v] : uniform);
}

// joint tables, edge-id order with caller strides -> position order [MS][MS]
template <int MS>
__global__ void k_gather_joint(const float *__restrict__ jin, uint32_t rs, uint64_t es,
                               const uint32_t *__restrict__ pos_edge, const uint32_t *__restrict__ in_src,
                               const uint32_t *__restrict__ dst_of_edge, const uint8_t *__restrict__ node_s,
                               uint32_t uniform, uint32_t E, float *__restrict__ jout) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t p = t / (MS * MS);
    if (p >= E) return;
    int k = (int)(t % (MS * MS));
    int i = k / MS, j = k % MS;
    uint32_t e = pos_edge[p];
    int x = uniform ? (int)uniform : node_s[in_src[p]];
    int y = uniform ? (int)uniform : node_s[dst_of_edge[e]];
    float v = 0.0f;
    if (i < x && j < y) v = jin[(uint64_t)e * es + (uint64_t)i * rs + j];
    jout[p * (MS * MS) + k] = v;
}

// beliefs [V][ld] <-> [V][MS] (zero beyond S_v)
__global__ void k_beliefs_in(const float *__restrict__ in, uint32_t ld, uint32_t V, uint32_t ms,
                             const uint8_t *__restrict__ node_s, uint32_t uniform, const uint32_t *__restrict__ perm,
                             float *__restrict__ b) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t v = t / ms;
    if (v >= V) return;
    uint32_t i = (uint32_t)(t % ms);
    uint32_t s = uniform ? uniform : node_s[v];
    const uint64_t row = perm ? perm[v] : v;
    b[t] = (i < s) ? in[row * ld + i] : 0.0f;
}

__global__ void k_beliefs_out(const float *__restrict__ b, uint32_t ld, uint32_t V, uint32_t ms,
                              const uint8_t *__restrict__ node_s, uint32_t uniform, const uint32_t *__restrict__ perm,
                              float *__restrict__ out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t v = t / ms;
    if (v >= V) return;
    uint32_t i = (uint32_t)(t % ms);
    uint32_t s = uniform ? uniform : node_s[v];
    const uint64_t row = perm ? perm[v] : v;
    if (i < ld && i < s) out[row * ld + i] = b[t];
}

// out-degree histogram and the renumbering by decreasing out-degree
// histogram of node ids: the lanes of a warp holding the same id add their
// count with one atomic (edge lists grouped by source, and a power-law
// graph's hubs, otherwise queue thousands of atomics on one address)
__global__ void k_out_degree(const uint32_t *__restrict__ src, uint32_t E, uint32_t *__restrict__ deg) {
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t key = e < E ? src[e] : 0xffffffffu;
    const unsigned same = __match_any_sync(0xffffffffu, key);
    if (e < E && (threadIdx.x & 31u) == (unsigned)(__ffs(same) - 1)) atomicAdd(deg + key, (unsigned)__popc(same));
}

// sort keys: decreasing out-degree; with indeg, then increasing in-degree
// (both clamped to 16 bits), so the 32 nodes of a warp have similar in-degrees
// and the node pass's per-node loops diverge less
__global__ void k_degree_keys(uint32_t *__restrict__ deg, const uint32_t *__restrict__ indeg, uint32_t V,
                              uint32_t *__restrict__ iota) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    if (indeg) deg[v] = ((0xffffu - min(deg[v], 0xffffu)) << 16) | min(indeg[v], 0xffffu);
    else deg[v] = 0xffffffffu - deg[v];
    iota[v] = (uint32_t)v;
}

// number of sorted keys below `limit` (the keys of out-degree >= 2 nodes)
__global__ void k_count_reused(const uint32_t *__restrict__ keys, uint32_t V, uint32_t limit, uint32_t *__restrict__ out) {
    uint32_t lo = 0, hi = V;
    while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if (keys[mid] < limit) lo = mid + 1;
        else hi = mid;
    }
    *out = lo;
}

// renumbering breaks out-degree ties by in-degree unless BP_REORDER_INDEG=0:
// on the 16.8M-node power-law graph k_flood went from 0.902 to 0.879 ms per
// iteration (the same clocks), since a warp's per-node loops over in-edges
// then run about as long in every lane
static bool reorder_by_indegree() {
    const char *env = getenv("BP_REORDER_INDEG");
    return !(env && env[0] == '0');
}

__global__ void k_invert_perm(const uint32_t *__restrict__ new_to_old, uint32_t V, uint32_t *__restrict__ old_to_new) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < V) old_to_new[new_to_old[i]] = (uint32_t)i;
}

__global__ void k_relabel(const uint32_t *__restrict__ in, uint64_t n, const uint32_t *__restrict__ old_to_new,
                          uint32_t *__restrict__ out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = old_to_new[in[i]];
}

__global__ void k_permute_u8(const uint8_t *__restrict__ in, const uint32_t *__restrict__ new_to_old, uint32_t V,
                             uint8_t *__restrict__ out) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < V) out[i] = in[new_to_old[i]];
}

// messages [E][ld] edge-id order <-> [E][MS] position order (zero beyond x)
__global__ void k_messages_in(const float *__restrict__ in, uint32_t ld, uint32_t E, uint32_t ms,
                              const uint32_t *__restrict__ pos_edge, const uint32_t *__restrict__ in_src,
                              const uint8_t *__restrict__ node_s, uint32_t uniform, float *__restrict__ m) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t p = t / ms;
    if (p >= E) return;
    uint32_t i = (uint32_t)(t % ms);
    uint32_t x = uniform ? uniform : node_s[in_src[p]];
    uint32_t e = pos_edge[p];
    m[t] = (i < x && i < ld) ? in[(uint64_t)e * ld + i] : 0.0f;
}

__global__ void k_messages_out(const float *__restrict__ m, uint32_t ld, uint32_t E, uint32_t ms,
                               const uint32_t *__restrict__ pos_edge, const uint32_t *__restrict__ in_src,
                               const uint8_t *__restrict__ node_s, uint32_t uniform, float *__restrict__ out) {
    uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t p = t / ms;
    if (p >= E) return;
    uint32_t i = (uint32_t)(t % ms);
    uint32_t x = uniform ? uniform : node_s[in_src[p]];
    uint32_t e = pos_edge[p];
    if (i < x && i < ld) out[(uint64_t)e * ld + i] = m[t];
}

__global__ void k_validate_edges(const uint32_t *__restrict__ src, const uint32_t *__restrict__ dst,
                                 uint32_t E, uint32_t V, uint32_t *__restrict__ bad) {
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < E && (src[e] >= V || dst[e] >= V)) atomicOr(bad, 1u);
}

__global__ void k_iota(uint32_t *__restrict__ a, uint32_t n) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = (uint32_t)i;
}

// position -> destination node
__global__ void k_pos_dst(const uint32_t *__restrict__ ptr, uint32_t V, uint32_t *__restrict__ pos_dst) {
    uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    for (uint32_t p = ptr[v]; p < ptr[v + 1]; ++p) pos_dst[p] = (uint32_t)v;
}

__global__ void k_src_of_edges(const uint32_t *__restrict__ edge_pos, const uint32_t *__restrict__ in_src,
                               uint32_t E, uint32_t *__restrict__ src_e, uint32_t *__restrict__ iota) {
    uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= E) return;
    src_e[e] = in_src[edge_pos[e]];
    iota[e] = (uint32_t)e;
}

__global__ void k_out_arrays(const uint32_t *__restrict__ out_edges, const uint32_t *__restrict__ edge_pos,
                             const uint32_t *__restrict__ pos_dst, uint32_t E, uint32_t *__restrict__ out_pos,
                             uint32_t *__restrict__ out_dst) {
    uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= E) return;
    uint32_t p = edge_pos[out_edges[q]];
    out_pos[q] = p;
    out_dst[q] = pos_dst[p];
}

static int bits_for(uint32_t n) {
    int b = 1;
    while (b < 32 && (1ull << b) < (uint64_t)n) ++b;
    return b;
}

// stable sort of (key, value) pairs by key, device memory
// ptr[V + 1] from E keys sorted ascending, all below V (see k_run_ends)
static int fill_ptr_from_sorted(bp_graph *g, const uint32_t *keys, uint32_t E, uint32_t V, uint32_t *ptr) {
    BP_CUDA(cudaMemsetAsync(ptr, 0, sizeof(uint32_t), g->stream));
    if (V == 0) return BP_OK;
    uint32_t *end = nullptr;
    BP_CUDA(cudaMallocAsync((void **)&end, sizeof(uint32_t) * V, g->stream));
    BP_CUDA(cudaMemsetAsync(end, 0, sizeof(uint32_t) * V, g->stream));
    if (E) k_run_ends<<<grid_for(E, 256), 256, 0, g->stream>>>(keys, E, end);
    BP_CUDA(cudaGetLastError());
    size_t temp = 0;
    BP_CUDA(cub::DeviceScan::InclusiveScan(nullptr, temp, end, ptr + 1, MaxU32(), (int64_t)V, g->stream));
    void *tmp = nullptr;
    BP_CUDA(cudaMallocAsync(&tmp, temp, g->stream));
    cudaError_t e = cub::DeviceScan::InclusiveScan(tmp, temp, end, ptr + 1, MaxU32(), (int64_t)V, g->stream);
    cudaFreeAsync(tmp, g->stream);
    cudaFreeAsync(end, g->stream);
    if (e != cudaSuccess) return cuda_fail(e, "DeviceScan::InclusiveScan", __FILE__, __LINE__);
    return BP_OK;
}

template <typename T>
static int radix_sort_pairs(bp_graph *g, const uint32_t *keys_in, uint32_t *keys_out,
                            const T *vals_in, T *vals_out, uint32_t n, uint32_t key_range) {
    if (n == 0) return BP_OK;
    size_t temp = 0;
    int end_bit = bits_for(key_range + 1);
    BP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, keys_in, keys_out, vals_in, vals_out, (int64_t)n, 0,
                                            end_bit, g->stream));
    void *tmp = nullptr;
    BP_CUDA(cudaMallocAsync(&tmp, temp, g->stream));
    cudaError_t e = cub::DeviceRadixSort::SortPairs(tmp, temp, keys_in, keys_out, vals_in, vals_out, (int64_t)n, 0,
                                                    end_bit, g->stream);
    cudaFreeAsync(tmp, g->stream);
    if (e != cudaSuccess) return cuda_fail(e, "DeviceRadixSort::SortPairs", __FILE__, __LINE__);
    return BP_OK;
}

template <int MS, bool UNI>
static int launch_gather_joint(bp_graph *g, const float *jin, uint32_t rs, uint64_t es, const uint32_t *dst_e) {
    uint64_t n = (uint64_t)g->E * MS * MS;
    if (n == 0) return BP_OK;
    k_gather_joint<MS><<<grid_for(n, 256), 256, 0, g->stream>>>(jin, rs, es, g->pos_edge, g->in_src, dst_e,
                                                                 g->node_s, g->uniform, g->E, g->joint);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

static int gather_joint(bp_graph *g, const float *jin, uint32_t rs, uint64_t es, const uint32_t *dst_e) {
    BP_DISPATCH_MS(g->ms, true, launch_gather_joint, g, jin, rs, es, dst_e);
}

// copy a host or device array to a device buffer that this call owns
static int to_device(bp_graph *g, const void *src, size_t bytes, int memory, void **dev, bool *owned) {
    if (memory == BP_MEM_DEVICE) {
        *dev = const_cast<void *>(src);
        *owned = false;
        return BP_OK;
    }
    BP_CUDA(cudaMallocAsync(dev, bytes ? bytes : 16, g->stream));
    *owned = true;
    if (bytes) BP_CUDA(cudaMemcpyAsync(*dev, src, bytes, cudaMemcpyHostToDevice, g->stream));
    return BP_OK;
}

int ensure_host_in_ptr(bp_graph *g) {
    if (g->in_ptr_host) return BP_OK;
    g->in_ptr_host = (uint32_t *)malloc(sizeof(uint32_t) * ((size_t)g->V + 1));
    if (!g->in_ptr_host) return set_error(BP_ERR_NOMEM, "host allocation failed");
    BP_CUDA(cudaMemcpyAsync(g->in_ptr_host, g->in_ptr, sizeof(uint32_t) * ((size_t)g->V + 1),
                            cudaMemcpyDeviceToHost, g->stream));
    BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

// src-sorted CSR for the tree schedule: out-edges of a node in insertion
// order (graph.c:249-283), as positions and destination nodes
// the inverse of pos_edge, for the callers that walk edges in id order (the
// source-sorted CSR, the edge schedule); a graph build skips it: its scatter
// of E 4-byte stores at random positions cost more DRAM traffic than any
// other step of the build
int ensure_edge_pos(bp_graph *g) {
    if (g->edge_pos || g->E == 0) return BP_OK;
    int st;
    if ((st = dev_alloc(g, (void **)&g->edge_pos, sizeof(uint32_t) * (size_t)g->E))) return st;
    k_invert_perm<<<grid_for(g->E, 256), 256, 0, g->stream>>>(g->pos_edge, g->E, g->edge_pos);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

int ensure_out_csr(bp_graph *g) {
    if (g->out_ptr) return BP_OK;
    int st;
    if ((st = ensure_edge_pos(g))) return st;
    uint32_t E = g->E, V = g->V;
    if ((st = dev_alloc(g, (void **)&g->out_ptr, sizeof(uint32_t) * ((size_t)V + 1)))) return st;
    if ((st = dev_alloc(g, (void **)&g->out_pos, sizeof(uint32_t) * (size_t)E))) return st;
    if ((st = dev_alloc(g, (void **)&g->out_dst, sizeof(uint32_t) * (size_t)E))) return st;
    if ((st = dev_alloc(g, (void **)&g->pos_dst, sizeof(uint32_t) * (size_t)E))) return st;
    k_pos_dst<<<grid_for(V, 256), 256, 0, g->stream>>>(g->in_ptr, V, g->pos_dst);
    BP_CUDA(cudaGetLastError());
    uint32_t *src_e = nullptr, *iota = nullptr, *keys = nullptr, *order = nullptr;
    BP_CUDA(cudaMallocAsync((void **)&src_e, sizeof(uint32_t) * (E ? E : 1), g->stream));
    BP_CUDA(cudaMallocAsync((void **)&iota, sizeof(uint32_t) * (E ? E : 1), g->stream));
    BP_CUDA(cudaMallocAsync((void **)&keys, sizeof(uint32_t) * (E ? E : 1), g->stream));
    BP_CUDA(cudaMallocAsync((void **)&order, sizeof(uint32_t) * (E ? E : 1), g->stream));
    if (E) {
        k_src_of_edges<<<grid_for(E, 256), 256, 0, g->stream>>>(g->edge_pos, g->in_src, E, src_e, iota);
        BP_CUDA(cudaGetLastError());
    }
    if ((st = radix_sort_pairs(g, src_e, keys, iota, order, E, V))) return st;
    if ((st = fill_ptr_from_sorted(g, keys, E, V, g->out_ptr))) return st;
    if (E) {
        k_out_arrays<<<grid_for(E, 256), 256, 0, g->stream>>>(order, g->edge_pos, g->pos_dst, E, g->out_pos,
                                                              g->out_dst);
        BP_CUDA(cudaGetLastError());
    }
    cudaFreeAsync(src_e, g->stream);
    cudaFreeAsync(iota, g->stream);
    cudaFreeAsync(keys, g->stream);
    cudaFreeAsync(order, g->stream);
    BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

// ---- split flooding schedule layout (used by loopy.cu) ---------------------

// per position: the range of its source (the sort key)
__global__ void k_split_keys(const uint32_t *__restrict__ in_src, uint32_t E, uint32_t range_nodes,
                             uint32_t *__restrict__ key) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p < E) key[p] = in_src[p] / range_nodes;
}

// the send-order streams and the inverse permutation
template <int MS>
__global__ void k_split_gather(const uint32_t *__restrict__ s_pos, uint32_t E, const uint32_t *__restrict__ in_src,
                               const uint32_t *__restrict__ pos_edge, const float *__restrict__ joint,
                               uint32_t *__restrict__ s_src, uint32_t *__restrict__ s_edge,
                               uint32_t *__restrict__ s_inv, float *__restrict__ s_joint) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= E) return;
    const uint32_t p = s_pos[k];
    s_src[k] = in_src[p];
    s_edge[k] = pos_edge[p];
    s_inv[p] = (uint32_t)k;
    float j[MS * MS];
    ldv<MS * MS>(joint + (size_t)p * (MS * MS), j);
    stv<MS * MS>(s_joint + (size_t)k * (MS * MS), j);
}

void split_free(bp_graph *g) {
    auto &s = g->split;
    void *ptrs[] = {s.s_src, s.s_edge, s.s_pos, s.s_inv, s.s_joint, s.s_msg[0], s.s_msg[1]};
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, g->stream);
    s = bp_graph::Split{};
}

template <int MS>
static int split_gather(bp_graph *g) {
    auto &s = g->split;
    k_split_gather<MS><<<grid_for(g->E, 256), 256, 0, g->stream>>>(s.s_pos, g->E, g->in_src, g->pos_edge, g->joint,
                                                                   s.s_src, s.s_edge, s.s_inv, s.s_joint);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

int split_build(bp_graph *g, uint32_t range_nodes) {
    auto &s = g->split;
    if (s.state) return BP_OK;
    const uint32_t V = g->V, E = g->E, ms = g->ms;
    s.state = -1;
    if (!g->uniform || ms > 4 || V == 0 || E == 0 || range_nodes == 0) return BP_OK;
    StageTrace trace(g->stream, "split layout");
    const uint32_t R = (uint32_t)(((uint64_t)V + range_nodes - 1) / range_nodes);
    s.R = R;
    s.range_nodes = range_nodes;
    int st;
    if ((st = dev_alloc(g, (void **)&s.s_src, sizeof(uint32_t) * (size_t)E))) return st;
    if ((st = dev_alloc(g, (void **)&s.s_edge, sizeof(uint32_t) * (size_t)E))) return st;
    if ((st = dev_alloc(g, (void **)&s.s_pos, sizeof(uint32_t) * (size_t)E))) return st;
    if ((st = dev_alloc(g, (void **)&s.s_inv, sizeof(uint32_t) * (size_t)E))) return st;
    if ((st = dev_alloc(g, (void **)&s.s_joint, sizeof(float) * ms * ms * (size_t)E))) return st;
    for (int k = 0; k < 2; ++k)
        if ((st = dev_alloc(g, (void **)&s.s_msg[k], sizeof(float) * ms * (size_t)E))) return st;
    trace.mark("allocate");
    uint32_t *key = nullptr, *key_sorted = nullptr, *iota = nullptr;
    BP_CUDA(cudaMallocAsync((void **)&key, sizeof(uint32_t) * E, g->stream));
    BP_CUDA(cudaMallocAsync((void **)&key_sorted, sizeof(uint32_t) * E, g->stream));
    BP_CUDA(cudaMallocAsync((void **)&iota, sizeof(uint32_t) * E, g->stream));
    k_split_keys<<<grid_for(E, 256), 256, 0, g->stream>>>(g->in_src, E, range_nodes, key);
    k_iota<<<grid_for(E, 256), 256, 0, g->stream>>>(iota, E);
    BP_CUDA(cudaGetLastError());
    // stable: inside a range the positions stay in order
    if ((st = radix_sort_pairs(g, key, key_sorted, iota, s.s_pos, E, R - 1))) return st;
    trace.mark("range sort");
    switch (ms) {
    case 1: st = split_gather<1>(g); break;
    case 2: st = split_gather<2>(g); break;
    case 3: st = split_gather<3>(g); break;
    default: st = split_gather<4>(g); break;
    }
    if (st) return st;
    cudaFreeAsync(key, g->stream);
    cudaFreeAsync(key_sorted, g->stream);
    cudaFreeAsync(iota, g->stream);
    trace.mark("gather");
    s.state = 1;
    return BP_OK;
}

static void free_graph(bp_graph *g) {
    if (!g) return;
    void *ptrs[] = {g->new_to_old, g->in_ptr, g->in_src, g->pos_edge, g->edge_pos, g->pos_dims, g->node_s, g->joint,
                    g->belief, g->msg[0], g->msg[1], g->q[0], g->q[1], g->out_ptr, g->out_pos,
                    g->out_dst, g->pos_dst, g->partials, g->absdiff, g->ctl, g->visited, g->staging,
                    g->run_len, g->run_s};
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, g->stream);
    split_free(g);
    tree_clear(g);
    for (auto &c : g->loop_graph)
        if (c.exec) cudaGraphExecDestroy(c.exec);
    if (g->stream) cudaStreamSynchronize(g->stream);
    release_pinned_ctl(g->ctl_host);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
    free(g->node_s_host);
    free(g->in_ptr_host);
    delete g;
}

static int create_impl(bp_graph *g, const bp_graph_desc *d) {
    const uint32_t V = d->num_nodes, E = d->num_edges;
    int st;
    StageTrace trace(g->stream, "create");
    // ---- state counts (validated on the host when they are host memory)
    std::vector<uint32_t> s32;
    const uint32_t *states = d->node_num_states;
    uint32_t smax = 0, smin = 0xffffffffu;
    if (!states) {
        if (d->uniform_states < 1 || d->uniform_states > BP_MAX_STATES)
            return set_error(BP_ERR_SHAPE, "uniform_states %u not in [1, %d]", d->uniform_states, BP_MAX_STATES);
        smax = smin = d->uniform_states;
    } else {
        if (d->memory == BP_MEM_DEVICE) {
            s32.resize(V);
            if (V) BP_CUDA(cudaMemcpy(s32.data(), states, sizeof(uint32_t) * V, cudaMemcpyDeviceToHost));
            states = s32.data();
        }
        for (uint32_t v = 0; v < V; ++v) {
            if (states[v] < 1 || states[v] > BP_MAX_STATES)
                return set_error(BP_ERR_SHAPE, "node %u has %u states (must be 1..%d)", v, states[v], BP_MAX_STATES);
            smax = std::max(smax, states[v]);
            smin = std::min(smin, states[v]);
        }
        if (V == 0) smax = smin = 1;
    }
    g->ms = smax;
    g->uniform = (smax == smin) ? smax : 0;
    g->node_s_host = (uint8_t *)malloc(V ? V : 1);
    if (!g->node_s_host) return set_error(BP_ERR_NOMEM, "host allocation failed");
    if (states)
        for (uint32_t v = 0; v < V; ++v) g->node_s_host[v] = (uint8_t)states[v];
    else
        memset(g->node_s_host, (int)d->uniform_states, V);
    trace.mark("state counts");

    // ---- device arrays
    const size_t ms = g->ms;
    // padding past the ends: the staged iteration kernel copies whole node
    // tiles and 16-byte-aligned ranges (loopy.cu)
    if ((st = dev_alloc(g, (void **)&g->in_ptr, sizeof(uint32_t) * ((size_t)V + 1 + kArrayPadNodes)))) return st;
    if ((st = dev_alloc(g, (void **)&g->in_src, sizeof(uint32_t) * ((size_t)E + kArrayPadEdges)))) return st;
    if ((st = dev_alloc(g, (void **)&g->pos_edge, sizeof(uint32_t) * (size_t)E))) return st;
    // edge_pos (position of each edge id) is built on first use (ensure_edge_pos)
    if ((st = dev_alloc(g, (void **)&g->node_s, (size_t)V))) return st;
    if (!g->uniform && (st = dev_alloc(g, (void **)&g->pos_dims, (size_t)E))) return st;
    if ((st = dev_alloc(g, (void **)&g->joint, sizeof(float) * ms * ms * ((size_t)E + kArrayPadEdges)))) return st;
    if ((st = dev_alloc(g, (void **)&g->belief, sizeof(float) * ms * ((size_t)V + kArrayPadNodes)))) return st;
    for (int k = 0; k < 2; ++k) {
        if ((st = dev_alloc(g, (void **)&g->msg[k], sizeof(float) * ms * ((size_t)E + kArrayPadEdges)))) return st;
        if ((st = dev_alloc(g, (void **)&g->q[k], sizeof(float) * ms * (size_t)V))) return st;
        BP_CUDA(cudaMemsetAsync(g->msg[k], 0, sizeof(float) * ms * (size_t)E, g->stream));
        BP_CUDA(cudaMemsetAsync(g->q[k], 0, sizeof(float) * ms * (size_t)V, g->stream));
    }
    BP_CUDA(cudaMemsetAsync(g->belief, 0, sizeof(float) * ms * (size_t)V, g->stream));
    if ((st = dev_alloc(g, (void **)&g->ctl, sizeof(bpx::LoopyCtl)))) return st;
    g->ctl_host = pinned_ctl();
    if (!g->ctl_host) return set_error(BP_ERR_NOMEM, "pinned host allocation failed");
    if ((st = dev_alloc(g, (void **)&g->visited, (size_t)V))) return st;
    BP_CUDA(cudaMemsetAsync(g->visited, 0, (size_t)V, g->stream));
    trace.mark("allocate + clear");

    // state counts -> u8
    {
        void *s_dev = nullptr;
        bool owned = false;
        if (d->node_num_states) {
            if ((st = to_device(g, d->node_num_states, sizeof(uint32_t) * V, d->memory, &s_dev, &owned))) return st;
        }
        if (V) {
            k_states_u8<<<grid_for(V, 256), 256, 0, g->stream>>>((const uint32_t *)s_dev, V, d->uniform_states,
                                                                g->node_s);
            BP_CUDA(cudaGetLastError());
        }
        if (owned) cudaFreeAsync(s_dev, g->stream);
    }

    // ---- joint tables of a host graph: upload on a side stream while the
    // edges are sorted on the graph's stream
    void *jd = nullptr;
    bool own_j = false;
    cudaStream_t side = nullptr;
    cudaEvent_t joint_ready = nullptr;
    size_t jbytes = 0;
    if (E) {
        const uint32_t rs = d->joint_row_stride;
        const uint64_t es = d->joint_edge_stride;
        if (rs < g->ms || es < (uint64_t)rs * (g->ms - 1) + g->ms)
            return set_error(BP_ERR_SHAPE, "joint strides (%u, %llu) too small for %u states", rs,
                             (unsigned long long)es, g->ms);
        jbytes = sizeof(float) * (es * (uint64_t)(E - 1) + (uint64_t)rs * (g->ms - 1) + g->ms);
        if (d->memory == BP_MEM_HOST) {
            BP_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
            BP_CUDA(cudaEventCreateWithFlags(&joint_ready, cudaEventDisableTiming));
            BP_CUDA(cudaMallocAsync(&jd, jbytes, side));
            BP_CUDA(cudaMemcpyAsync(jd, d->edge_joint, jbytes, cudaMemcpyHostToDevice, side));
            BP_CUDA(cudaEventRecord(joint_ready, side));
            own_j = true;
        } else {
            jd = const_cast<float *>(d->edge_joint);
        }
    }

    // ---- edges
    void *src = nullptr, *dst = nullptr;
    bool own_src = false, own_dst = false;
    if ((st = to_device(g, d->edge_src, sizeof(uint32_t) * (size_t)E, d->memory, &src, &own_src))) return st;
    if ((st = to_device(g, d->edge_dst, sizeof(uint32_t) * (size_t)E, d->memory, &dst, &own_dst))) return st;
    if (E) {
        uint32_t *bad = nullptr;
        BP_CUDA(cudaMallocAsync((void **)&bad, sizeof(uint32_t), g->stream));
        BP_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), g->stream));
        k_validate_edges<<<grid_for(E, 256), 256, 0, g->stream>>>((const uint32_t *)src, (const uint32_t *)dst, E,
                                                                  V, bad);
        BP_CUDA(cudaGetLastError());
        uint32_t hbad = 0;
        BP_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
        BP_CUDA(cudaStreamSynchronize(g->stream));
        cudaFreeAsync(bad, g->stream);
        if (hbad) {
            if (own_src) cudaFreeAsync(src, g->stream);
            if (own_dst) cudaFreeAsync(dst, g->stream);
            return set_error(BP_ERR_INVALID, "an edge endpoint is >= num_nodes (%u)", V);
        }
    }
    trace.mark("edges in + validate");


    if (d->flags & BP_GRAPH_REORDER_BY_OUT_DEGREE) {
        if (d->dest_node_list) return set_error(BP_ERR_INVALID, "renumbering ignores a caller CSR: pass none");
        // internal id = rank by (out-degree descending, in-degree ascending,
        // id ascending)
        uint32_t *deg = nullptr, *iota = nullptr, *keys = nullptr, *old_to_new = nullptr;
        BP_CUDA(cudaMallocAsync((void **)&deg, sizeof(uint32_t) * (V ? V : 1), g->stream));
        BP_CUDA(cudaMallocAsync((void **)&iota, sizeof(uint32_t) * (V ? V : 1), g->stream));
        BP_CUDA(cudaMallocAsync((void **)&keys, sizeof(uint32_t) * (V ? V : 1), g->stream));
        BP_CUDA(cudaMallocAsync((void **)&old_to_new, sizeof(uint32_t) * (V ? V : 1), g->stream));
        if ((st = dev_alloc(g, (void **)&g->new_to_old, sizeof(uint32_t) * (size_t)V))) return st;
        trace.mark("renumber: allocate");
        BP_CUDA(cudaMemsetAsync(deg, 0, sizeof(uint32_t) * V, g->stream));
        if (E) k_out_degree<<<grid_for(E, 256), 256, 0, g->stream>>>((const uint32_t *)src, E, deg);
        const bool by_in = reorder_by_indegree();
        if (by_in) {
            // the in-degree histogram in old_to_new (filled later)
            BP_CUDA(cudaMemsetAsync(old_to_new, 0, sizeof(uint32_t) * V, g->stream));
            if (E) k_out_degree<<<grid_for(E, 256), 256, 0, g->stream>>>((const uint32_t *)dst, E, old_to_new);
        }
        if (V) k_degree_keys<<<grid_for(V, 256), 256, 0, g->stream>>>(deg, by_in ? old_to_new : nullptr, V, iota);
        BP_CUDA(cudaGetLastError());
        if (V) {
            size_t temp = 0;
            BP_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, temp, deg, keys, iota, g->new_to_old, (int64_t)V, 0, 32,
                                                    g->stream));
            void *tmp = nullptr;
            BP_CUDA(cudaMallocAsync(&tmp, temp, g->stream));
            cudaError_t se = cub::DeviceRadixSort::SortPairs(tmp, temp, deg, keys, iota, g->new_to_old, (int64_t)V, 0,
                                                             32, g->stream);
            cudaFreeAsync(tmp, g->stream);
            if (se != cudaSuccess) return cuda_fail(se, "DeviceRadixSort::SortPairs", __FILE__, __LINE__);
            k_invert_perm<<<grid_for(V, 256), 256, 0, g->stream>>>(g->new_to_old, V, old_to_new);
            k_count_reused<<<1, 1, 0, g->stream>>>(keys, V, by_in ? 0xfffe0000u : 0xfffffffeu, deg);
            BP_CUDA(cudaMemcpyAsync(&g->reuse_nodes, deg, sizeof(uint32_t), cudaMemcpyDeviceToHost, g->stream));
        }
        trace.mark("renumber: degree sort");
        uint32_t *src2 = nullptr, *dst2 = nullptr;
        BP_CUDA(cudaMallocAsync((void **)&src2, sizeof(uint32_t) * (E ? E : 1), g->stream));
        BP_CUDA(cudaMallocAsync((void **)&dst2, sizeof(uint32_t) * (E ? E : 1), g->stream));
        if (E) {
            k_relabel<<<grid_for(E, 256), 256, 0, g->stream>>>((const uint32_t *)src, E, old_to_new, src2);
            k_relabel<<<grid_for(E, 256), 256, 0, g->stream>>>((const uint32_t *)dst, E, old_to_new, dst2);
        }
        if (V) {
            uint8_t *s8 = nullptr;
            BP_CUDA(cudaMallocAsync((void **)&s8, V, g->stream));
            k_permute_u8<<<grid_for(V, 256), 256, 0, g->stream>>>(g->node_s, g->new_to_old, V, s8);
            BP_CUDA(cudaMemcpyAsync(g->node_s, s8, V, cudaMemcpyDeviceToDevice, g->stream));
            cudaFreeAsync(s8, g->stream);
            if (!g->uniform) {
                BP_CUDA(cudaMemcpyAsync(g->node_s_host, g->node_s, V, cudaMemcpyDeviceToHost, g->stream));
                BP_CUDA(cudaStreamSynchronize(g->stream));
            }
        }
        BP_CUDA(cudaGetLastError());
        cudaFreeAsync(deg, g->stream);
        cudaFreeAsync(iota, g->stream);
        cudaFreeAsync(keys, g->stream);
        cudaFreeAsync(old_to_new, g->stream);
        if (own_src) cudaFreeAsync(src, g->stream);
        if (own_dst) cudaFreeAsync(dst, g->stream);
        src = src2;
        dst = dst2;
        own_src = own_dst = true;
        trace.mark("renumber");
    }

    if (d->dest_node_list && d->dest_edge_list) {
        // the caller's dest-CSR (struct graph's dest_nodes_to_edges_*)
        void *nl = nullptr, *el = nullptr;
        bool own_nl = false, own_el = false;
        if ((st = to_device(g, d->dest_node_list, sizeof(uint32_t) * V, d->memory, &nl, &own_nl))) return st;
        if ((st = to_device(g, d->dest_edge_list, sizeof(uint32_t) * (size_t)E, d->memory, &el, &own_el))) return st;
        k_ptr_from_node_list<<<grid_for((uint64_t)V + 1, 256), 256, 0, g->stream>>>((const uint32_t *)nl, V, E,
                                                                                     g->in_ptr);
        BP_CUDA(cudaGetLastError());
        if (E) BP_CUDA(cudaMemcpyAsync(g->pos_edge, el, sizeof(uint32_t) * (size_t)E, cudaMemcpyDeviceToDevice,
                                       g->stream));
        if (own_nl) cudaFreeAsync(nl, g->stream);
        if (own_el) cudaFreeAsync(el, g->stream);
    } else {
        // stable sort of (source, edge id) by destination
        uint64_t *vals = nullptr, *vals_sorted = nullptr;
        uint32_t *keys = nullptr;
        BP_CUDA(cudaMallocAsync((void **)&vals, sizeof(uint64_t) * (E ? E : 1), g->stream));
        BP_CUDA(cudaMallocAsync((void **)&vals_sorted, sizeof(uint64_t) * (E ? E : 1), g->stream));
        BP_CUDA(cudaMallocAsync((void **)&keys, sizeof(uint32_t) * (E ? E : 1), g->stream));
        if (E) {
            k_pack_src_id<<<grid_for(E, 256), 256, 0, g->stream>>>((const uint32_t *)src, E, vals);
            BP_CUDA(cudaGetLastError());
        }
        if ((st = radix_sort_pairs(g, (const uint32_t *)dst, keys, (const uint64_t *)vals, vals_sorted, E, V)))
            return st;
        if ((st = fill_ptr_from_sorted(g, keys, E, V, g->in_ptr))) return st;
        if (E) {
            k_unpack_positions<<<grid_for(E, 256), 256, 0, g->stream>>>(vals_sorted, keys, E, g->node_s, g->in_src,
                                                                        g->pos_edge, g->pos_dims);
            BP_CUDA(cudaGetLastError());
        }
        cudaFreeAsync(vals, g->stream);
        cudaFreeAsync(vals_sorted, g->stream);
        cudaFreeAsync(keys, g->stream);
    }
    trace.mark("dest sort");
    if (E && d->dest_node_list && d->dest_edge_list) {
        k_positions<<<grid_for(E, 256), 256, 0, g->stream>>>(g->pos_edge, (const uint32_t *)src,
                                                             (const uint32_t *)dst, E, g->node_s, g->in_src,
                                                             g->pos_dims);
        BP_CUDA(cudaGetLastError());
    }

    // ---- joint tables: edge-id order with the caller's strides -> position order
    if (E) {
        if (joint_ready) BP_CUDA(cudaStreamWaitEvent(g->stream, joint_ready, 0));
        if ((st = gather_joint(g, (const float *)jd, d->joint_row_stride, d->joint_edge_stride,
                               (const uint32_t *)dst)))
            return st;
        if (own_j) cudaFreeAsync(jd, g->stream);
    }
    trace.mark("positions + joint");
    if (joint_ready) cudaEventDestroy(joint_ready);
    if (side) cudaStreamDestroy(side);
    if (own_src) cudaFreeAsync(src, g->stream);
    if (own_dst) cudaFreeAsync(dst, g->stream);
    BP_CUDA(cudaEventCreate(&g->ev0));
    BP_CUDA(cudaEventCreate(&g->ev1));
    // large uniform graphs: the split flooding schedule's second edge order
    if ((st = flood_split_prepare(g))) return st;
    BP_CUDA(cudaStreamSynchronize(g->stream));
    trace.mark("finish");
    return BP_OK;
}

}  // namespace bpx

using namespace bpx;

extern "C" {

int bp_version(void) { return 1; }

const char *bp_last_error(void) { return bpx::g_last_error; }

const char *bp_status_string(int status) {
    switch (status) {
    case BP_OK: return "ok";
    case BP_ERR_INVALID: return "invalid argument";
    case BP_ERR_SHAPE: return "shape out of range";
    case BP_ERR_CUDA: return "CUDA error";
    case BP_ERR_NOMEM: return "out of device memory";
    case BP_ERR_NO_DEVICE: return "no CUDA device";
    case BP_ERR_GRAPH: return "graph has nodes unreachable from the tree seed set";
    case BP_ERR_STATE: return "call out of order";
    case BP_ERR_TIMEOUT: return "bounded device wait timed out";
    default: return "unknown status";
    }
}

int bp_graph_create(bp_graph **out, const bp_graph_desc *d, void *stream) {
    if (!out || !d) return set_error(BP_ERR_INVALID, "null argument");
    *out = nullptr;
    if (d->num_edges && (!d->edge_src || !d->edge_dst || !d->edge_joint))
        return set_error(BP_ERR_INVALID, "edge arrays missing");
    if (d->memory != BP_MEM_HOST && d->memory != BP_MEM_DEVICE)
        return set_error(BP_ERR_INVALID, "memory must be BP_MEM_HOST or BP_MEM_DEVICE");
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) return set_error(BP_ERR_NO_DEVICE, "no CUDA device available");
    bp_graph *g = new bp_graph();
    cudaGetDevice(&g->device);
    ensure_pool(g->device);
    g->V = d->num_nodes;
    g->E = d->num_edges;
    if (stream) {
        g->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete g;
            return set_error(BP_ERR_CUDA, "cudaStreamCreate failed");
        }
        g->own_stream = true;
    }
    int st = create_impl(g, d);
    if (st != BP_OK) {
        char keep[512];
        snprintf(keep, sizeof keep, "%s", bp_last_error());
        free_graph(g);
        set_error(st, "%s", keep);
        return st;
    }
    *out = g;
    return BP_OK;
}

void bp_graph_destroy(bp_graph *g) {
    if (!g) return;
    if (g->stream) cudaStreamSynchronize(g->stream);
    free_graph(g);
}

int bp_release_cached_memory(void) {
    int dev = 0;
    BP_CUDA(cudaGetDevice(&dev));
    cudaMemPool_t pool;
    BP_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    BP_CUDA(cudaDeviceSynchronize());
    BP_CUDA(cudaMemPoolTrimTo(pool, 0));
    return BP_OK;
}

int bp_reserve_cached_memory(uint64_t bytes) {
    int dev = 0;
    BP_CUDA(cudaGetDevice(&dev));
    ensure_pool(dev);
    cudaMemPool_t pool;
    BP_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t held = 0;
    BP_CUDA(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &held));
    if (held >= bytes) return BP_OK;
    cudaStream_t st = nullptr;
    BP_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes - held, pool, st);
    if (e == cudaSuccess) e = cudaFreeAsync(p, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    if (e != cudaSuccess) return cuda_fail(e, "reserving pool memory", __FILE__, __LINE__);
    return BP_OK;
}

int bp_graph_info(const bp_graph *g, uint32_t *V, uint32_t *E, uint32_t *ms, uint32_t *uni) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    if (V) *V = g->V;
    if (E) *E = g->E;
    if (ms) *ms = g->ms;
    if (uni) *uni = g->uniform;
    return BP_OK;
}

int bp_graph_device_bytes(const bp_graph *g, uint64_t *bytes) {
    if (!g || !bytes) return set_error(BP_ERR_INVALID, "null argument");
    *bytes = g->device_bytes;
    return BP_OK;
}

int bp_set_stream(bp_graph *g, void *stream) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    BP_CUDA(cudaStreamSynchronize(g->stream));
    if (g->own_stream) cudaStreamDestroy(g->stream);
    g->own_stream = false;
    if (stream) {
        g->stream = (cudaStream_t)stream;
    } else {
        BP_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
        g->own_stream = true;
    }
    return BP_OK;
}

int bp_synchronize(bp_graph *g) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

// ---- beliefs / messages --------------------------------------------------
static int staged_in(bp_graph *g, const float *src, size_t bytes, int memory, const float **dev) {
    if (memory == BP_MEM_DEVICE) {
        *dev = src;
        return BP_OK;
    }
    int st = ensure_staging(g, bytes);
    if (st) return st;
    if (bytes) BP_CUDA(cudaMemcpyAsync(g->staging, src, bytes, cudaMemcpyHostToDevice, g->stream));
    *dev = g->staging;
    return BP_OK;
}

int bp_set_beliefs(bp_graph *g, const float *b, uint32_t ld, int memory) {
    if (!g || (!b && g->V)) return set_error(BP_ERR_INVALID, "null argument");
    if (ld < g->ms) return set_error(BP_ERR_SHAPE, "ld %u < max states %u", ld, g->ms);
    if (g->V == 0) return BP_OK;
    const float *dev = nullptr;
    int st = staged_in(g, b, sizeof(float) * (size_t)ld * g->V, memory, &dev);
    if (st) return st;
    uint64_t n = (uint64_t)g->V * g->ms;
    k_beliefs_in<<<grid_for(n, 256), 256, 0, g->stream>>>(dev, ld, g->V, g->ms, g->node_s, g->uniform, g->new_to_old,
                                                          g->belief);
    BP_CUDA(cudaGetLastError());
    if (memory == BP_MEM_HOST) BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

int bp_get_beliefs(bp_graph *g, float *b, uint32_t ld, int memory) {
    if (!g || (!b && g->V)) return set_error(BP_ERR_INVALID, "null argument");
    if (g->V == 0) return BP_OK;
    uint64_t n = (uint64_t)g->V * g->ms;
    if (memory == BP_MEM_DEVICE) {
        k_beliefs_out<<<grid_for(n, 256), 256, 0, g->stream>>>(g->belief, ld, g->V, g->ms, g->node_s, g->uniform,
                                                               g->new_to_old, b);
        BP_CUDA(cudaGetLastError());
        return BP_OK;
    }
    if (ld == g->ms && !g->new_to_old) {
        BP_CUDA(cudaMemcpyAsync(b, g->belief, sizeof(float) * n, cudaMemcpyDeviceToHost, g->stream));
        BP_CUDA(cudaStreamSynchronize(g->stream));
        return BP_OK;
    }
    size_t bytes = sizeof(float) * (size_t)ld * g->V;
    int st = ensure_staging(g, bytes);
    if (st) return st;
    // keep the caller's slots beyond each node's state count intact
    BP_CUDA(cudaMemcpyAsync(g->staging, b, bytes, cudaMemcpyHostToDevice, g->stream));
    k_beliefs_out<<<grid_for(n, 256), 256, 0, g->stream>>>(g->belief, ld, g->V, g->ms, g->node_s, g->uniform,
                                                           g->new_to_old, g->staging);
    BP_CUDA(cudaGetLastError());
    BP_CUDA(cudaMemcpyAsync(b, g->staging, bytes, cudaMemcpyDeviceToHost, g->stream));
    BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

int bp_set_messages(bp_graph *g, int slot, const float *m, uint32_t ld, int memory) {
    if (!g || (!m && g->E) || slot < 0 || slot > 1) return set_error(BP_ERR_INVALID, "bad argument");
    if (g->E == 0) return BP_OK;
    const float *dev = nullptr;
    int st = staged_in(g, m, sizeof(float) * (size_t)ld * g->E, memory, &dev);
    if (st) return st;
    uint64_t n = (uint64_t)g->E * g->ms;
    k_messages_in<<<grid_for(n, 256), 256, 0, g->stream>>>(dev, ld, g->E, g->ms, g->pos_edge, g->in_src, g->node_s,
                                                           g->uniform, g->msg[slot]);
    BP_CUDA(cudaGetLastError());
    if (memory == BP_MEM_HOST) BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

int bp_get_messages(bp_graph *g, int slot, float *m, uint32_t ld, int memory) {
    if (!g || (!m && g->E) || slot < 0 || slot > 1) return set_error(BP_ERR_INVALID, "bad argument");
    if (g->E == 0) return BP_OK;
    uint64_t n = (uint64_t)g->E * g->ms;
    if (memory == BP_MEM_DEVICE) {
        k_messages_out<<<grid_for(n, 256), 256, 0, g->stream>>>(g->msg[slot], ld, g->E, g->ms, g->pos_edge, g->in_src,
                                                                g->node_s, g->uniform, m);
        BP_CUDA(cudaGetLastError());
        return BP_OK;
    }
    size_t bytes = sizeof(float) * (size_t)ld * g->E;
    int st = ensure_staging(g, bytes);
    if (st) return st;
    BP_CUDA(cudaMemcpyAsync(g->staging, m, bytes, cudaMemcpyHostToDevice, g->stream));
    k_messages_out<<<grid_for(n, 256), 256, 0, g->stream>>>(g->msg[slot], ld, g->E, g->ms, g->pos_edge, g->in_src,
                                                            g->node_s, g->uniform, g->staging);
    BP_CUDA(cudaGetLastError());
    BP_CUDA(cudaMemcpyAsync(m, g->staging, bytes, cudaMemcpyDeviceToHost, g->stream));
    BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

int bp_set_latest_slot(bp_graph *g, int slot) {
    if (!g || slot < 0 || slot > 1) return set_error(BP_ERR_INVALID, "bad argument");
    g->latest = slot;
    return BP_OK;
}

int bp_get_latest_slot(const bp_graph *g, int *slot) {
    if (!g || !slot) return set_error(BP_ERR_INVALID, "bad argument");
    *slot = g->latest;
    return BP_OK;
}

int bp_set_visited(bp_graph *g, const char *visited) {
    if (!g || (!visited && g->V)) return set_error(BP_ERR_INVALID, "bad argument");
    if (g->V) BP_CUDA(cudaMemcpyAsync(g->visited, visited, g->V, cudaMemcpyHostToDevice, g->stream));
    BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

int bp_get_visited(bp_graph *g, char *visited) {
    if (!g || (!visited && g->V)) return set_error(BP_ERR_INVALID, "bad argument");
    if (g->V) BP_CUDA(cudaMemcpyAsync(visited, g->visited, g->V, cudaMemcpyDeviceToHost, g->stream));
    BP_CUDA(cudaStreamSynchronize(g->stream));
    return BP_OK;
}

}  // extern "C"
