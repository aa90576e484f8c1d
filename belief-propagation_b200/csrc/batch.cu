// batch.cu -- many independent networks in one persistent launch.
//
// Each network runs the reference's loopy_propagate_until (graph.c:1278-1324)
// with its own stopping rule.  A network is small enough (thousands of nodes)
// that one thread block can own it for its whole run: the block takes the
// next network from a work queue (networks sorted by work, largest first),
// iterates it to convergence with block-wide barriers between the send and
// marginalise phases, writes its results, and takes the next one.  No grid
// barrier and no host round trip per iteration: a whole batch is one launch
// per state count, captured together in a CUDA graph.  The per-value
// arithmetic is the plain engine's (bp_device.cuh), so every network's
// beliefs, messages and iteration count equal what bp_loopy gives for it.
//
// Layout: the networks' arrays are concatenated (network order); inside a
// network the edges are destination-sorted exactly as in bp_graph.
#include <errno.h>
#include <stdio.h>
#include <sys/stat.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "bp_device.cuh"
#include "bp_serial.cuh"
#include "bp_internal.h"

namespace bpx {

struct NetInfo {
    uint32_t V, E, S, pad;
    uint64_t node_off;   // into belief/q (floats): sum of V*S before
    uint64_t edge_off;   // into in_src / pos_edge (edges)
    uint64_t msg_off;    // into msg / absdiff (floats): sum of E*S before
    uint64_t joint_off;  // into joint (floats): sum of E*S*S before
    uint64_t ptr_off;    // into in_ptr: sum of (V+1) before
};

struct NetResult {
    uint32_t iterations, executed, converged, latest;
    float delta, prev_delta;
    double delta_d;
};

struct BatchArgs {
    const NetInfo *info;
    const uint32_t *in_ptr, *in_src, *pos_edge;
    const float *joint;
    float *belief, *msg0, *msg1, *q0, *q1, *absdiff;
    uint64_t ad_stride;   // floats between the two |diff| buffers (by iteration parity)
    uint32_t sum_ch;      // serial mode: staging chunk of the block's serial sum (dynamic smem 2 sum_ch floats)
    NetResult *res;
    uint8_t *latest;
    float tol;
    uint32_t max_it;
    int serial, init;
};

// the reference's serial fp32 sum of x[0, n) (graph.c:1300-1309), one thread
__device__ __noinline__ float net_serial_sum(const float *x, uint64_t n) {
    float s = 0.0f;
    uint64_t k = 0;
    for (; k + 4 <= n; k += 4) {
        const float t0 = x[k], t1 = x[k + 1], t2 = x[k + 2], t3 = x[k + 3];
        s = FADD(s, t0);
        s = FADD(s, t1);
        s = FADD(s, t2);
        s = FADD(s, t3);
    }
    for (; k < n; ++k) s = FADD(s, x[k]);
    return s;
}

// the same sum by the whole block: thread 0 adds in order out of shared
// memory while threads 32.. stage the next ch terms (buf: 2 ch floats,
// ch % 4 == 0); with fewer than 64 threads thread 0 reads global memory
// itself.  Every thread calls it and gets the sum.
__device__ float net_serial_sum_block(const float *x, uint64_t n, float *buf, uint32_t ch, float *s_res) {
    const uint32_t T = blockDim.x, tid = threadIdx.x;
    __syncthreads();   // buf and *s_res are free
    if (T < 64 || ch == 0) {
        if (tid == 0) *s_res = net_serial_sum(x, n);
    } else {
        const uint64_t nch = (n + ch - 1) / ch;
        auto stage = [&](uint64_t c) {
            const uint64_t base = c * ch;
            const uint32_t cnt = (uint32_t)min((uint64_t)ch, n - base);
            float *dst = buf + (c & 1) * ch;
            for (uint32_t k = tid - 32; k < cnt; k += T - 32) dst[k] = x[base + k];
        };
        if (tid >= 32 && nch) stage(0);
        __syncthreads();
        float s = 0.0f;
        for (uint64_t c = 0; c < nch; ++c) {
            if (tid >= 32) {
                if (c + 1 < nch) stage(c + 1);
            } else if (tid == 0) {
                const uint32_t cnt = (uint32_t)min((uint64_t)ch, n - c * ch);
                const float *b = buf + (c & 1) * ch;
                uint32_t k = 0;
                for (; k + 4 <= cnt; k += 4) {
                    const float4 v = *reinterpret_cast<const float4 *>(b + k);
                    s = FADD(s, v.x);
                    s = FADD(s, v.y);
                    s = FADD(s, v.z);
                    s = FADD(s, v.w);
                }
                for (; k < cnt; ++k) s = FADD(s, b[k]);
            }
            __syncthreads();
        }
        if (tid == 0) *s_res = s;
    }
    __syncthreads();
    const float r = *s_res;
    __syncthreads();
    return r;
}

template <int S, bool SER>
__device__ void solve_network(const BatchArgs &a, uint32_t n, double *red, int *s_flag, double *s_tot, float *s_res,
                              float *sbuf) {
    const NetInfo ni = a.info[n];
    const uint32_t V = ni.V, E = ni.E;
    const uint32_t *ptr = a.in_ptr + ni.ptr_off;
    const uint32_t *src = a.in_src + ni.edge_off;
    const float *J = a.joint + ni.joint_off;
    float *b = a.belief + ni.node_off;
    float *msg[2] = {a.msg0 + ni.msg_off, a.msg1 + ni.msg_off};
    float *q[2] = {a.q0 + ni.node_off, a.q1 + ni.node_off};
    const uint32_t T = blockDim.x, tid = threadIdx.x;
    int latest = a.latest[n];

    if (a.init) {  // init_previous_edge (graph.c:725-751)
        for (uint32_t p = tid; p < E; p += T) {
            float buf[S], m[S];
            ldv<S>(b + (size_t)src[p] * S, buf);
            send_msg<S, true>(J + (size_t)p * S * S, buf, S, S, m);
            stv<S>(msg[latest] + (size_t)p * S, m);
        }
        __syncthreads();
    }
    // Q_1 = b * prod of the latest messages (graph.c:860-882)
    for (uint32_t v = tid; v < V; v += T) {
        float bb[S];
        ldv<S>(b + (size_t)v * S, bb);
        for (uint32_t p = ptr[v]; p < ptr[v + 1]; ++p) {
            float mm[S];
            ldv<S>(msg[latest] + (size_t)p * S, mm);
            combine<S, true>(bb, mm, S);
        }
        stv<S>(q[0] + (size_t)v * S, bb);
    }
    __syncthreads();

    float prev_f = -1.0f, delta_f = 0.0f;
    double prev_d = -1.0, delta_d = 0.0;
    // serial delta (thread 0): intervals of the serial sums of this check and
    // of the previous one, whether each is the sum itself, and their buffers
    double d_lo = 0.0, d_hi = 0.0, p_lo = -1.0, p_hi = -1.0;
    bool d_ex = true, p_ex = true, d_ref = false, p_ref = false;
    // the narrowed interval needs 3 floats of staging per thread
    const bool refine_ok = blockDim.x <= 1024 && 3u * blockDim.x <= 2u * a.sum_ch;
    uint32_t d_buf = 0, p_buf = 0;
    const uint64_t nterms = (uint64_t)E * S;
    const float *ad_base = SER ? a.absdiff + ni.msg_off : nullptr;
    uint32_t it = 0, ret = a.max_it, converged = 0;
    for (it = 0; it < a.max_it; ++it) {
        const float *m_old = msg[latest];
        float *m_new = msg[latest ^ 1];
        const float *q_in = q[it & 1];
        float *q_out = q[(it + 1) & 1];
        double dsum = 0.0;
        for (uint32_t p = tid; p < E; p += T) {
            float qq[S], m[S], o[S];
            ldv<S>(q_in + (size_t)src[p] * S, qq);
            ldv<S>(m_old + (size_t)p * S, o);
            send_msg<S, true>(J + (size_t)p * S * S, qq, S, S, m);
            float ad[S];
#pragma unroll
            for (int k = 0; k < S; ++k) {
                float d = FSUB(o[k], m[k]);
                if (d != d) d = 0.0f;
                ad[k] = fabsf(d);
                dsum += (double)ad[k];
            }
            if constexpr (SER)
                stv<S>(a.absdiff + (size_t)(it & 1u) * a.ad_stride + ni.msg_off +
                           (size_t)a.pos_edge[ni.edge_off + p] * S,
                       ad);
            stv<S>(m_new + (size_t)p * S, m);
        }
        __syncthreads();
        for (uint32_t v = tid; v < V; v += T) {
            const uint32_t r0 = ptr[v], r1 = ptr[v + 1];
            float prod[S], bb[S];
#pragma unroll
            for (int i = 0; i < S; ++i) prod[i] = 1.0f;
            for (uint32_t p = r0; p < r1; ++p) {
                float mm[S];
                ldv<S>(m_new + (size_t)p * S, mm);
                combine<S, true>(prod, mm, S);
            }
            ldv<S>(b + (size_t)v * S, bb);
            if (r1 > r0) {
#pragma unroll
                for (int i = 0; i < S; ++i) bb[i] = FMUL(bb[i], prod[i]);
            }
            normalise<S, true>(bb, S);
            stv<S>(b + (size_t)v * S, bb);
            float qo[S];
#pragma unroll
            for (int i = 0; i < S; ++i) qo[i] = bb[i];
            for (uint32_t p = r0; p < r1; ++p) {
                float mm[S];
                ldv<S>(m_new + (size_t)p * S, mm);
                combine<S, true>(qo, mm, S);
            }
            stv<S>(q_out + (size_t)v * S, qo);
        }
        // delta and the stopping rule (graph.c:1300-1318)
        double tot = 0.0;
        {
            double v = warp_sum(dsum);
            const int lane = tid & 31, w = tid >> 5;
            if (lane == 0) red[w] = v;
            __syncthreads();
            if (w == 0) {
                double t = lane < (int)(T >> 5) ? red[lane] : 0.0;
                tot = warp_sum(t);
            }
        }
        if constexpr (SER) {
            // every thread takes the same decision: the f64 sum to all, the
            // reference's serial fp32 decision from its interval, and the
            // serial sums (formed by the whole block) only where it straddles
            if (tid == 0) *s_tot = tot;
            __syncthreads();
            tot = *s_tot;
            double lo, hi;
            serial_interval(tot, nterms, lo, hi);
            bool s_ex = false, s_ref = false;
            float s = (float)tot;
            int d = serial_decide(lo, hi, false, p_lo, p_hi, p_ex, a.tol);
            const float *ad_cur = ad_base + (size_t)(it & 1u) * a.ad_stride;
            const float *ad_prev = ad_base + (size_t)p_buf * a.ad_stride;
            // narrowed from the terms' own rounding errors (intersected with
            // the bound; an interval holding one float gives the sum)
            auto narrow = [&](double &L, double &H, bool &ex, float &val, double l2, double h2) {
                L = fmax(L, l2);
                H = fmin(H, h2);
                float f;
                if (interval_pins(L, H, f)) {
                    L = H = (double)f;
                    ex = true;
                    val = f;
                }
            };
            if (d < 0 && refine_ok) {
                double l2, h2;
                if (refine_block<1024>(ad_cur, nterms, sbuf, 2 * a.sum_ch, l2, h2)) narrow(lo, hi, s_ex, s, l2, h2);
                s_ref = true;
                d = serial_decide(lo, hi, s_ex, p_lo, p_hi, p_ex, a.tol);
                if (d < 0 && !p_ex && !p_ref) {
                    if (refine_block<1024>(ad_prev, nterms, sbuf, 2 * a.sum_ch, l2, h2))
                        narrow(p_lo, p_hi, p_ex, prev_f, l2, h2);
                    p_ref = true;
                    d = serial_decide(lo, hi, s_ex, p_lo, p_hi, p_ex, a.tol);
                }
            }
            if (d < 0 && !s_ex) {
                s = net_serial_sum_block(ad_cur, nterms, sbuf, a.sum_ch, s_res);
                lo = hi = (double)s;
                s_ex = true;
                d = serial_decide(lo, hi, true, p_lo, p_hi, p_ex, a.tol);
            }
            if (d < 0) {
                prev_f = net_serial_sum_block(ad_prev, nterms, sbuf, a.sum_ch, s_res);
                p_lo = p_hi = (double)prev_f;
                p_ex = true;
                d = serial_decide(lo, hi, true, p_lo, p_hi, true, a.tol);
            }
            delta_f = s;
            delta_d = tot;
            d_lo = lo;
            d_hi = hi;
            d_ex = s_ex;
            d_ref = s_ref;
            d_buf = it & 1u;
            const bool stop = d == 1;
            if (stop) {
                ret = it;
                converged = 1;
            } else if (it < a.max_it - 1) {
                prev_f = delta_f;
                prev_d = delta_d;
                p_lo = d_lo;
                p_hi = d_hi;
                p_ex = d_ex;
                p_ref = d_ref;
                p_buf = d_buf;
            }
            latest ^= 1;
            __syncthreads();   // *s_tot is rewritten next iteration
            if (stop) break;
            continue;
        }
        if (tid == 0) {
            delta_d = tot;
            delta_f = (float)tot;
            const bool stop = (tot < (double)a.tol) || (fabs(tot - prev_d) < (double)a.tol);
            if (stop) {
                ret = it;
                converged = 1;
            } else if (it < a.max_it - 1) {
                prev_f = delta_f;
                prev_d = delta_d;
            }
            *s_flag = stop ? 1 : 0;
        }
        __syncthreads();
        latest ^= 1;
        const int stop = *s_flag;
        __syncthreads();
        if (stop) break;
    }
    // the returned delta and previous delta where the loop decided without
    // forming them (the whole block; every thread has the same flags)
    if (SER && !d_ex) delta_f = net_serial_sum_block(ad_base + (size_t)d_buf * a.ad_stride, nterms, sbuf, a.sum_ch, s_res);
    if (SER && !p_ex) prev_f = net_serial_sum_block(ad_base + (size_t)p_buf * a.ad_stride, nterms, sbuf, a.sum_ch, s_res);
    if (tid == 0) {
        NetResult r;
        r.iterations = converged ? ret : a.max_it;
        r.executed = converged ? it + 1 : a.max_it;
        r.converged = converged;
        r.latest = (uint32_t)latest;
        r.delta = delta_f;
        r.prev_delta = prev_f;
        r.delta_d = delta_d;
        a.res[n] = r;
        a.latest[n] = (uint8_t)latest;
    }
    __syncthreads();
}

template <int S, bool SER>
__global__ void k_batch_solve(const BatchArgs a, const uint32_t *__restrict__ order, uint32_t count,
                              uint32_t *queue) {
    __shared__ double red[32];
    __shared__ int s_flag;
    __shared__ uint32_t s_next;
    __shared__ double s_tot;
    __shared__ float s_res;
    extern __shared__ __align__(16) float sbuf[];   // serial mode: 2 sum_ch floats
    for (;;) {
        if (threadIdx.x == 0) s_next = atomicAdd(queue, 1u);
        __syncthreads();
        const uint32_t k = s_next;
        __syncthreads();
        if (k >= count) break;
        solve_network<S, SER>(a, order[k], red, &s_flag, &s_tot, &s_res, sbuf);
    }
}

// beliefs / messages between the caller's concatenated layout and ours
__global__ void k_batch_msgs_out(const float *__restrict__ m0, const float *__restrict__ m1,
                                 const uint8_t *__restrict__ latest, const NetInfo *__restrict__ info,
                                 const uint32_t *__restrict__ pos_edge, const uint32_t *__restrict__ net_of_edge,
                                 uint64_t total_edges, float *__restrict__ out) {
    const uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total_edges) return;
    const uint32_t n = net_of_edge[g];
    const NetInfo ni = info[n];
    const uint64_t p = g - ni.edge_off;
    const float *m = (latest[n] ? m1 : m0) + ni.msg_off;
    const uint64_t e = pos_edge[g];
    for (uint32_t k = 0; k < ni.S; ++k) out[ni.msg_off + e * ni.S + k] = m[p * ni.S + k];
}

struct Group {
    int S = 0;
    uint32_t vmax = 0;             // networks of at most vmax nodes; 0: the larger ones
    std::vector<uint32_t> order;   // network ids, largest work first
    uint32_t *d_order = nullptr;
    uint32_t block = 0;            // threads per block (0 = not tuned yet)
    uint32_t grid = 0;
};

}  // namespace bpx

struct bp_batch {
    uint32_t N = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<bpx::NetInfo> info;
    uint64_t totV = 0, totE = 0, totNodeF = 0, totMsgF = 0, totJointF = 0, totPtr = 0;
    bpx::NetInfo *d_info = nullptr;
    uint32_t *in_ptr = nullptr, *in_src = nullptr, *pos_edge = nullptr, *net_of_edge = nullptr;
    float *joint = nullptr, *belief = nullptr, *msg[2] = {nullptr, nullptr}, *q[2] = {nullptr, nullptr};
    float *absdiff = nullptr, *staging = nullptr;
    bpx::NetResult *res = nullptr;
    uint8_t *latest = nullptr;
    uint32_t *queues = nullptr;   // one counter per group
    std::vector<bpx::Group> groups;
    cudaGraphExec_t exec = nullptr;
    uint64_t exec_key = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int sm_count = 148;
    std::vector<cudaStream_t> side;     // per-group streams
    std::vector<cudaEvent_t> side_ev;
    cudaEvent_t fork_ev = nullptr;
};

namespace bpx {

template <int S>
static int launch_group(bp_batch *bt, Group &gr, const BatchArgs &a, uint32_t gi, uint32_t block, uint32_t grid,
                        cudaStream_t s) {
    if (a.serial)
        k_batch_solve<S, true><<<grid, block, sizeof(float) * 2 * a.sum_ch, s>>>(a, gr.d_order,
                                                                               (uint32_t)gr.order.size(), bt->queues + gi);
    else
        k_batch_solve<S, false><<<grid, block, 0, s>>>(a, gr.d_order, (uint32_t)gr.order.size(), bt->queues + gi);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

static int launch_group_s(bp_batch *bt, Group &gr, const BatchArgs &a, uint32_t gi, uint32_t block, uint32_t grid,
                          cudaStream_t s) {
    switch (gr.S) {
    case 1: return launch_group<1>(bt, gr, a, gi, block, grid, s);
    case 2: return launch_group<2>(bt, gr, a, gi, block, grid, s);
    case 3: return launch_group<3>(bt, gr, a, gi, block, grid, s);
    case 4: return launch_group<4>(bt, gr, a, gi, block, grid, s);
    case 5: return launch_group<5>(bt, gr, a, gi, block, grid, s);
    case 6: return launch_group<6>(bt, gr, a, gi, block, grid, s);
    case 7: return launch_group<7>(bt, gr, a, gi, block, grid, s);
    case 8: return launch_group<8>(bt, gr, a, gi, block, grid, s);
    case 9: return launch_group<9>(bt, gr, a, gi, block, grid, s);
    default: return launch_group<10>(bt, gr, a, gi, block, grid, s);
    }
}

constexpr uint32_t kSumChunk = 1024;   // serial mode: 8 KB of dynamic shared memory per block

// networks of at most this many nodes form a group of their own per state
// count (BP_BATCH_SMALL_NODES; default 0: one group per state count).  On
// the 4096-network batch (f64 delta) a bound of 512 nodes measured 35.2-35.5k
// networks/s against 35.8-35.9k without; 256: 35.5k, 1024: 34.1k; serial
// delta 26.7k either way.  Tuned alone, the small groups still take 512
// threads per block: a small network's iteration is set by the block's
// barriers and reductions, not by its idle threads.
static uint32_t batch_small_nodes() {
    const char *env = getenv("BP_BATCH_SMALL_NODES");
    return env ? (uint32_t)strtoul(env, nullptr, 10) : 0u;
}

static BatchArgs batch_args(bp_batch *bt, float tol, uint32_t max_it, int serial, int init) {
    BatchArgs a;
    a.info = bt->d_info;
    a.in_ptr = bt->in_ptr;
    a.in_src = bt->in_src;
    a.pos_edge = bt->pos_edge;
    a.joint = bt->joint;
    a.belief = bt->belief;
    a.msg0 = bt->msg[0];
    a.msg1 = bt->msg[1];
    a.q0 = bt->q[0];
    a.q1 = bt->q[1];
    a.absdiff = bt->absdiff;
    a.sum_ch = serial ? kSumChunk : 0u;
    a.ad_stride = bt->totMsgF + 4;   // totMsgF % 4 == 0: buffer 1 keeps the 16-byte alignment of buffer 0
    a.res = bt->res;
    a.latest = bt->latest;
    a.tol = tol;
    a.max_it = max_it;
    a.serial = serial;
    a.init = init;
    return a;
}

// blocks that fit on the GPU at once for this group
template <int S>
static uint32_t occupancy_grid(bp_batch *bt, uint32_t block, size_t dyn) {
    int per_sm = 0;
    if (dyn) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_solve<S, true>, (int)block, dyn);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_solve<S, false>, (int)block, 0);
    if (per_sm < 1) per_sm = 1;
    return (uint32_t)per_sm * (uint32_t)bt->sm_count;
}

static uint32_t grid_for_group(bp_batch *bt, const Group &gr, uint32_t block, size_t dyn = 0) {
    uint32_t g = 0;
    switch (gr.S) {
    case 1: g = occupancy_grid<1>(bt, block, dyn); break;
    case 2: g = occupancy_grid<2>(bt, block, dyn); break;
    case 3: g = occupancy_grid<3>(bt, block, dyn); break;
    case 4: g = occupancy_grid<4>(bt, block, dyn); break;
    case 5: g = occupancy_grid<5>(bt, block, dyn); break;
    case 6: g = occupancy_grid<6>(bt, block, dyn); break;
    case 7: g = occupancy_grid<7>(bt, block, dyn); break;
    case 8: g = occupancy_grid<8>(bt, block, dyn); break;
    case 9: g = occupancy_grid<9>(bt, block, dyn); break;
    default: g = occupancy_grid<10>(bt, block, dyn); break;
    }
    return std::min<uint32_t>(g, (uint32_t)gr.order.size());
}

// the whole batched solve on bt->stream: reset queues, fork one stream per
// state-count group, launch each group's persistent kernel, join
static int enqueue_batch(bp_batch *bt, const BatchArgs &a) {
    BP_CUDA(cudaMemsetAsync(bt->queues, 0, sizeof(uint32_t) * bt->groups.size(), bt->stream));
    BP_CUDA(cudaEventRecord(bt->fork_ev, bt->stream));
    for (size_t gi = 0; gi < bt->groups.size(); ++gi) {
        Group &gr = bt->groups[gi];
        cudaStream_t s = bt->side[gi];
        BP_CUDA(cudaStreamWaitEvent(s, bt->fork_ev, 0));
        // serial mode holds 2 sum_ch floats of dynamic shared memory per block
        const uint32_t grid =
            a.sum_ch ? std::min(gr.grid, grid_for_group(bt, gr, gr.block, sizeof(float) * 2 * a.sum_ch)) : gr.grid;
        int st = launch_group_s(bt, gr, a, (uint32_t)gi, gr.block, grid, s);
        if (st) return st;
        BP_CUDA(cudaEventRecord(bt->side_ev[gi], s));
        BP_CUDA(cudaStreamWaitEvent(bt->stream, bt->side_ev[gi], 0));
    }
    return BP_OK;
}

static void batch_free(bp_batch *bt) {
    if (!bt) return;
    void *ptrs[] = {bt->d_info, bt->in_ptr, bt->in_src, bt->pos_edge, bt->net_of_edge, bt->joint, bt->belief,
                    bt->msg[0], bt->msg[1], bt->q[0], bt->q[1], bt->absdiff, bt->staging, bt->res,
                    bt->latest, bt->queues};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    for (auto &g : bt->groups)
        if (g.d_order) cudaFree(g.d_order);
    if (bt->exec) cudaGraphExecDestroy(bt->exec);
    for (auto s : bt->side) cudaStreamDestroy(s);
    for (auto e : bt->side_ev) cudaEventDestroy(e);
    if (bt->fork_ev) cudaEventDestroy(bt->fork_ev);
    if (bt->ev0) cudaEventDestroy(bt->ev0);
    if (bt->ev1) cudaEventDestroy(bt->ev1);
    if (bt->own_stream && bt->stream) cudaStreamDestroy(bt->stream);
    delete bt;
}

static int batch_create_impl(bp_batch *bt, uint32_t N, const bp_graph_desc *descs) {
    // ---- per-network sizes and the destination sort, on the host
    bt->info.resize(N);
    std::vector<uint32_t> h_ptr, h_src, h_pos, h_net;
    std::vector<float> h_joint;
    uint64_t node_f = 0, msg_f = 0, joint_f = 0, ptr_n = 0, edges = 0, nodes = 0;
    for (uint32_t n = 0; n < N; ++n) {
        const bp_graph_desc &d = descs[n];
        if (d.memory != BP_MEM_HOST) return set_error(BP_ERR_INVALID, "network %u: batch descriptors take host arrays", n);
        uint32_t S = d.uniform_states;
        if (d.node_num_states) {
            S = d.num_nodes ? d.node_num_states[0] : 1;
            for (uint32_t v = 0; v < d.num_nodes; ++v)
                if (d.node_num_states[v] != S)
                    return set_error(BP_ERR_SHAPE, "network %u: every node of a batched network needs the same "
                                                   "state count", n);
        }
        if (S < 1 || S > BP_MAX_STATES) return set_error(BP_ERR_SHAPE, "network %u: %u states", n, S);
        if (d.num_nodes == 0) return set_error(BP_ERR_SHAPE, "network %u has no nodes", n);
        if (d.joint_row_stride < S || d.joint_edge_stride < (uint64_t)d.joint_row_stride * (S - 1) + S)
            return set_error(BP_ERR_SHAPE, "network %u: joint strides too small", n);
        // every network's arrays start on a 16-byte boundary: the kernels load
        // S, S*S floats at a time as float2/float4 when S allows it
        node_f = (node_f + 3) & ~(uint64_t)3;
        msg_f = (msg_f + 3) & ~(uint64_t)3;
        joint_f = (joint_f + 3) & ~(uint64_t)3;
        h_joint.resize(joint_f, 0.0f);
        NetInfo &ni = bt->info[n];
        ni.V = d.num_nodes;
        ni.E = d.num_edges;
        ni.S = S;
        ni.pad = 0;
        ni.node_off = node_f;
        ni.edge_off = edges;
        ni.msg_off = msg_f;
        ni.joint_off = joint_f;
        ni.ptr_off = ptr_n;
        // stable counting sort by destination
        std::vector<uint32_t> cnt(ni.V + 1, 0);
        for (uint32_t e = 0; e < ni.E; ++e) {
            if (d.edge_src[e] >= ni.V || d.edge_dst[e] >= ni.V)
                return set_error(BP_ERR_INVALID, "network %u: edge %u endpoint out of range", n, e);
            cnt[d.edge_dst[e] + 1]++;
        }
        for (uint32_t v = 0; v < ni.V; ++v) cnt[v + 1] += cnt[v];
        h_ptr.insert(h_ptr.end(), cnt.begin(), cnt.end());
        std::vector<uint32_t> fill(cnt.begin(), cnt.end() - 1), perm(ni.E);
        for (uint32_t e = 0; e < ni.E; ++e) perm[fill[d.edge_dst[e]]++] = e;
        for (uint32_t p = 0; p < ni.E; ++p) {
            const uint32_t e = perm[p];
            h_src.push_back(d.edge_src[e]);
            h_pos.push_back(e);
            h_net.push_back(n);
            const float *t = d.edge_joint + (uint64_t)e * d.joint_edge_stride;
            for (uint32_t i = 0; i < S; ++i)
                for (uint32_t j = 0; j < S; ++j) h_joint.push_back(t[(uint64_t)i * d.joint_row_stride + j]);
        }
        node_f += (uint64_t)ni.V * S;
        msg_f += (uint64_t)ni.E * S;
        joint_f += (uint64_t)ni.E * S * S;
        ptr_n += ni.V + 1;
        edges += ni.E;
        nodes += ni.V;
    }
    node_f = (node_f + 3) & ~(uint64_t)3;
    msg_f = (msg_f + 3) & ~(uint64_t)3;
    for (const NetInfo &ni : bt->info)
        if ((ni.node_off | ni.msg_off | ni.joint_off) & 3u)
            return set_error(BP_ERR_STATE, "internal: unaligned network offsets");
    bt->totV = nodes;
    bt->totE = edges;
    bt->totNodeF = node_f;
    bt->totMsgF = msg_f;
    bt->totJointF = joint_f;
    bt->totPtr = ptr_n;

    auto alloc = [&](void **p, size_t bytes) -> int {
        BP_CUDA(cudaMalloc(p, bytes ? bytes : 16));
        return BP_OK;
    };
    int st;
    if ((st = alloc((void **)&bt->d_info, sizeof(NetInfo) * N))) return st;
    if ((st = alloc((void **)&bt->in_ptr, sizeof(uint32_t) * ptr_n))) return st;
    if ((st = alloc((void **)&bt->in_src, sizeof(uint32_t) * edges))) return st;
    if ((st = alloc((void **)&bt->pos_edge, sizeof(uint32_t) * edges))) return st;
    if ((st = alloc((void **)&bt->net_of_edge, sizeof(uint32_t) * edges))) return st;
    if ((st = alloc((void **)&bt->joint, sizeof(float) * joint_f))) return st;
    if ((st = alloc((void **)&bt->belief, sizeof(float) * node_f))) return st;
    for (int k = 0; k < 2; ++k) {
        if ((st = alloc((void **)&bt->msg[k], sizeof(float) * msg_f))) return st;
        if ((st = alloc((void **)&bt->q[k], sizeof(float) * node_f))) return st;
        BP_CUDA(cudaMemsetAsync(bt->msg[k], 0, sizeof(float) * msg_f, bt->stream));
    }
    if ((st = alloc((void **)&bt->res, sizeof(NetResult) * N))) return st;
    if ((st = alloc((void **)&bt->latest, N))) return st;
    BP_CUDA(cudaMemsetAsync(bt->latest, 1, N, bt->stream));
    BP_CUDA(cudaMemsetAsync(bt->belief, 0, sizeof(float) * node_f, bt->stream));
    BP_CUDA(cudaMemcpyAsync(bt->d_info, bt->info.data(), sizeof(NetInfo) * N, cudaMemcpyHostToDevice, bt->stream));
    BP_CUDA(cudaMemcpyAsync(bt->in_ptr, h_ptr.data(), sizeof(uint32_t) * ptr_n, cudaMemcpyHostToDevice, bt->stream));
    if (edges) {
        BP_CUDA(cudaMemcpyAsync(bt->in_src, h_src.data(), sizeof(uint32_t) * edges, cudaMemcpyHostToDevice, bt->stream));
        BP_CUDA(cudaMemcpyAsync(bt->pos_edge, h_pos.data(), sizeof(uint32_t) * edges, cudaMemcpyHostToDevice, bt->stream));
        BP_CUDA(cudaMemcpyAsync(bt->net_of_edge, h_net.data(), sizeof(uint32_t) * edges, cudaMemcpyHostToDevice,
                                bt->stream));
        BP_CUDA(cudaMemcpyAsync(bt->joint, h_joint.data(), sizeof(float) * joint_f, cudaMemcpyHostToDevice, bt->stream));
    }

    // ---- groups by state count and, optionally, size class (networks of
    // at most small_nodes nodes in a group with its own launch shape, queue
    // and stream)
    const uint32_t small_nodes = batch_small_nodes();
    auto work = [&](uint32_t n) {
        const NetInfo &x = bt->info[n];
        return (uint64_t)x.E * x.S * x.S + (uint64_t)x.V * x.S;
    };
    for (uint32_t n = 0; n < N; ++n) {
        const int S = (int)bt->info[n].S;
        const uint32_t vmax = (small_nodes && bt->info[n].V <= small_nodes) ? small_nodes : 0u;
        auto it = std::find_if(bt->groups.begin(), bt->groups.end(),
                               [&](const Group &g) { return g.S == S && g.vmax == vmax; });
        if (it == bt->groups.end()) {
            bt->groups.emplace_back();
            bt->groups.back().S = S;
            bt->groups.back().vmax = vmax;
            it = bt->groups.end() - 1;
        }
        it->order.push_back(n);
    }
    // the heaviest group is launched first
    std::vector<uint64_t> gwork(bt->groups.size(), 0);
    for (size_t gi = 0; gi < bt->groups.size(); ++gi)
        for (uint32_t n : bt->groups[gi].order) gwork[gi] += work(n);
    std::vector<size_t> gidx(bt->groups.size());
    std::iota(gidx.begin(), gidx.end(), 0);
    std::stable_sort(gidx.begin(), gidx.end(), [&](size_t x, size_t y) { return gwork[x] > gwork[y]; });
    {
        std::vector<Group> sorted;
        for (size_t i : gidx) sorted.push_back(std::move(bt->groups[i]));
        bt->groups = std::move(sorted);
    }
    for (auto &gr : bt->groups) {
        std::stable_sort(gr.order.begin(), gr.order.end(), [&](uint32_t x, uint32_t y) { return work(x) > work(y); });
        BP_CUDA(cudaMalloc((void **)&gr.d_order, sizeof(uint32_t) * gr.order.size()));
        BP_CUDA(cudaMemcpyAsync(gr.d_order, gr.order.data(), sizeof(uint32_t) * gr.order.size(),
                                cudaMemcpyHostToDevice, bt->stream));
        gr.block = 256;
        gr.grid = grid_for_group(bt, gr, gr.block);
        cudaStream_t s;
        BP_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        bt->side.push_back(s);
        cudaEvent_t e;
        BP_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        bt->side_ev.push_back(e);
    }
    if ((st = alloc((void **)&bt->queues, sizeof(uint32_t) * bt->groups.size()))) return st;
    BP_CUDA(cudaEventCreateWithFlags(&bt->fork_ev, cudaEventDisableTiming));
    BP_CUDA(cudaEventCreate(&bt->ev0));
    BP_CUDA(cudaEventCreate(&bt->ev1));
    BP_CUDA(cudaStreamSynchronize(bt->stream));
    return BP_OK;
}

// ---- autotuning of threads per block, cached on disk ---------------------
// kernel revision in the autotune key: a cached block size belongs to the
// kernel it was timed on
constexpr int kTuneRevision = 4;

static std::string tune_key(bp_batch *bt, const Group &gr, int serial) {
    uint64_t V = 0, E = 0;
    for (uint32_t n : gr.order) {
        V += bt->info[n].V;
        E += bt->info[n].E;
    }
    const uint64_t cnt = gr.order.size();
    const unsigned mv = (unsigned)(V / cnt), deg10 = (unsigned)(V ? 10 * E / V : 0);
    unsigned lv = 0;
    while ((1u << (lv + 1)) <= mv) ++lv;
    cudaDeviceProp prop;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaGetDeviceProperties(&prop, dev);
    char buf[512];
    snprintf(buf, sizeof buf, "%s|S=%d|vmax=%u|log2V=%u|deg10=%u|nets=%llu|delta=%s|rev=%d", prop.name, gr.S, gr.vmax,
             lv, deg10, (unsigned long long)(cnt >= 1024 ? 1024 : cnt), serial ? "serial" : "f64", kTuneRevision);
    for (char *c = buf; *c; ++c)
        if (*c == ' ') *c = '_';
    return buf;
}

static std::string cache_path() {
    const char *p = getenv("BP_AUTOTUNE_CACHE");
    if (p && *p) return p;
    const char *home = getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/bp_b200_autotune.txt";
}

// a cached (block, grid) for the key, or block 0
static uint32_t cache_lookup(const std::string &key, uint32_t *grid) {
    FILE *f = fopen(cache_path().c_str(), "r");
    if (!f) return 0;
    char line[1024], k[512];
    unsigned b = 0, gsz = 0, found = 0, found_g = 0;
    while (fgets(line, sizeof line, f))
        if (sscanf(line, "%511s %u %u", k, &b, &gsz) == 3 && key == k) {
            found = b;
            found_g = gsz;
        }
    fclose(f);
    *grid = found_g;
    return found;
}

// every directory on the way to `dir` (mkdir -p without a shell); false if
// one could not be made
static bool make_dirs(const std::string &dir) {
    for (size_t i = 1; i <= dir.size(); ++i) {
        if (i < dir.size() && dir[i] != '/') continue;
        const std::string part = dir.substr(0, i);
        if (mkdir(part.c_str(), 0755) != 0 && errno != EEXIST) return false;
    }
    return true;
}

static void cache_store(const std::string &key, uint32_t block, uint32_t grid) {
    std::string path = cache_path();
    const size_t slash = path.find_last_of('/');
    if (slash != std::string::npos && slash > 0 && !make_dirs(path.substr(0, slash))) return;
    FILE *f = fopen(path.c_str(), "a");
    if (!f) return;
    fprintf(f, "%s %u %u\n", key.c_str(), block, grid);
    fclose(f);
}

}  // namespace bpx

using namespace bpx;

extern "C" {

int bp_batch_create(bp_batch **out, uint32_t num_networks, const bp_graph_desc *descs, void *stream) {
    if (!out || (!descs && num_networks)) return set_error(BP_ERR_INVALID, "null argument");
    *out = nullptr;
    if (num_networks == 0) return set_error(BP_ERR_SHAPE, "empty batch");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(BP_ERR_NO_DEVICE, "no CUDA device");
    bp_batch *bt = new bp_batch();
    bt->N = num_networks;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&bt->sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (stream) {
        bt->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete bt;
            return set_error(BP_ERR_CUDA, "cudaStreamCreate failed");
        }
        bt->own_stream = true;
    }
    int st = batch_create_impl(bt, num_networks, descs);
    if (st) {
        char keep[512];
        snprintf(keep, sizeof keep, "%s", bp_last_error());
        batch_free(bt);
        set_error(st, "%s", keep);
        return st;
    }
    *out = bt;
    return BP_OK;
}

void bp_batch_destroy(bp_batch *bt) {
    if (!bt) return;
    cudaStreamSynchronize(bt->stream);
    batch_free(bt);
}

int bp_batch_layout(const bp_batch *bt, uint64_t *belief_offsets, uint64_t *message_offsets) {
    if (!bt) return set_error(BP_ERR_INVALID, "null batch");
    for (uint32_t n = 0; n < bt->N; ++n) {
        if (belief_offsets) belief_offsets[n] = bt->info[n].node_off;
        if (message_offsets) message_offsets[n] = bt->info[n].msg_off;
    }
    if (belief_offsets) belief_offsets[bt->N] = bt->totNodeF;
    if (message_offsets) message_offsets[bt->N] = bt->totMsgF;
    return BP_OK;
}

int bp_batch_set_beliefs(bp_batch *bt, const float *beliefs, int memory) {
    if (!bt || !beliefs) return set_error(BP_ERR_INVALID, "null argument");
    BP_CUDA(cudaMemcpyAsync(bt->belief, beliefs, sizeof(float) * bt->totNodeF,
                            memory == BP_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, bt->stream));
    BP_CUDA(cudaMemsetAsync(bt->latest, 1, bt->N, bt->stream));
    if (memory == BP_MEM_HOST) BP_CUDA(cudaStreamSynchronize(bt->stream));
    return BP_OK;
}

int bp_batch_get_beliefs(bp_batch *bt, float *beliefs, int memory) {
    if (!bt || !beliefs) return set_error(BP_ERR_INVALID, "null argument");
    BP_CUDA(cudaMemcpyAsync(beliefs, bt->belief, sizeof(float) * bt->totNodeF,
                            memory == BP_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, bt->stream));
    if (memory == BP_MEM_HOST) BP_CUDA(cudaStreamSynchronize(bt->stream));
    return BP_OK;
}

int bp_batch_get_messages(bp_batch *bt, float *messages, int memory) {
    if (!bt || !messages) return set_error(BP_ERR_INVALID, "null argument");
    if (bt->totE == 0) return BP_OK;
    float *dst = messages;
    if (memory == BP_MEM_HOST) {
        if (!bt->staging) BP_CUDA(cudaMalloc((void **)&bt->staging, sizeof(float) * bt->totMsgF));
        dst = bt->staging;
    }
    k_batch_msgs_out<<<grid_for(bt->totE, 256), 256, 0, bt->stream>>>(bt->msg[0], bt->msg[1], bt->latest, bt->d_info,
                                                                      bt->pos_edge, bt->net_of_edge, bt->totE, dst);
    BP_CUDA(cudaGetLastError());
    if (memory == BP_MEM_HOST) {
        BP_CUDA(cudaMemcpyAsync(messages, bt->staging, sizeof(float) * bt->totMsgF, cudaMemcpyDeviceToHost, bt->stream));
        BP_CUDA(cudaStreamSynchronize(bt->stream));
    }
    return BP_OK;
}

void bp_batch_default_options(bp_batch_options *o) {
    if (!o) return;
    o->tolerance = 1e-4f;
    o->max_iterations = 200;
    o->delta_mode = BP_DELTA_F64;
    o->block_threads = 0;
    o->init_messages = 1;
    o->reserved = 0;
}

int bp_batch_autotune(bp_batch *bt, const bp_batch_options *o) {
    if (!bt || !o) return set_error(BP_ERR_INVALID, "null argument");
    static const uint32_t cand[] = {64, 128, 256, 512};
    const int serial = o->delta_mode == BP_DELTA_SERIAL_F32;
    if (serial && !bt->absdiff) BP_CUDA(cudaMalloc((void **)&bt->absdiff, sizeof(float) * 2 * (bt->totMsgF + 4)));
    // beliefs are overwritten by trial runs: keep them
    float *keep = nullptr;
    BP_CUDA(cudaMalloc((void **)&keep, sizeof(float) * (bt->totNodeF + 1)));
    BP_CUDA(cudaMemcpyAsync(keep, bt->belief, sizeof(float) * bt->totNodeF, cudaMemcpyDeviceToDevice, bt->stream));
    std::vector<uint8_t> latest0(bt->N);
    BP_CUDA(cudaMemcpyAsync(latest0.data(), bt->latest, bt->N, cudaMemcpyDeviceToHost, bt->stream));
    BP_CUDA(cudaStreamSynchronize(bt->stream));
    const BatchArgs a = batch_args(bt, o->tolerance, o->max_iterations, serial, o->init_messages);
    for (size_t gi = 0; gi < bt->groups.size(); ++gi) {
        Group &gr = bt->groups[gi];
        const std::string key = tune_key(bt, gr, serial);
        uint32_t best_grid = 0;
        uint32_t best = cache_lookup(key, &best_grid);
        if (!best) {
            float best_ms = 1e30f;
            // block sizes, and networks in flight: a block keeps its
            // network's arrays in L2 across its iterations, so fewer blocks
            // than the GPU holds can be faster once the networks in flight
            // outgrow L2
            std::vector<std::pair<uint32_t, uint32_t>> trials;
            for (uint32_t c : cand) {
                const uint32_t occ = grid_for_group(bt, gr, c, sizeof(float) * 2 * a.sum_ch);
                trials.push_back({c, occ});
                for (uint32_t per_sm : {1u, 2u, 4u, 8u}) {
                    const uint32_t g = per_sm * (uint32_t)bt->sm_count;
                    if (g < occ) trials.push_back({c, g});
                }
            }
            for (const auto &tr : trials) {
                const uint32_t c = tr.first, grid = tr.second;
                float tot = 0.0f;
                for (int rep = 0; rep < 2; ++rep) {
                    BP_CUDA(cudaMemcpyAsync(bt->belief, keep, sizeof(float) * bt->totNodeF, cudaMemcpyDeviceToDevice,
                                            bt->stream));
                    BP_CUDA(cudaMemcpyAsync(bt->latest, latest0.data(), bt->N, cudaMemcpyHostToDevice, bt->stream));
                    BP_CUDA(cudaMemsetAsync(bt->queues + gi, 0, sizeof(uint32_t), bt->stream));
                    BP_CUDA(cudaEventRecord(bt->ev0, bt->stream));
                    int st = launch_group_s(bt, gr, a, (uint32_t)gi, c, grid, bt->stream);
                    if (st) {
                        cudaFree(keep);
                        return st;
                    }
                    BP_CUDA(cudaEventRecord(bt->ev1, bt->stream));
                    BP_CUDA(cudaEventSynchronize(bt->ev1));
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, bt->ev0, bt->ev1);
                    if (rep) tot += ms;
                }
                if (tot < best_ms) {
                    best_ms = tot;
                    best = c;
                    best_grid = grid;
                }
            }
            cache_store(key, best, best_grid);
        }
        gr.block = best;
        const uint32_t occ = grid_for_group(bt, gr, best);
        gr.grid = best_grid ? std::min(best_grid, occ) : occ;
    }
    BP_CUDA(cudaMemcpyAsync(bt->belief, keep, sizeof(float) * bt->totNodeF, cudaMemcpyDeviceToDevice, bt->stream));
    BP_CUDA(cudaMemcpyAsync(bt->latest, latest0.data(), bt->N, cudaMemcpyHostToDevice, bt->stream));
    BP_CUDA(cudaStreamSynchronize(bt->stream));
    cudaFree(keep);
    if (bt->exec) {
        cudaGraphExecDestroy(bt->exec);
        bt->exec = nullptr;
    }
    return BP_OK;
}

int bp_batch_get_groups(const bp_batch *bt, uint32_t *states, uint32_t *max_nodes, uint32_t *block, uint32_t *grid,
                        uint32_t *count) {
    if (!bt || !count) return set_error(BP_ERR_INVALID, "null argument");
    const uint32_t n = (uint32_t)bt->groups.size();
    for (uint32_t i = 0; i < n && i < *count; ++i) {
        if (states) states[i] = (uint32_t)bt->groups[i].S;
        if (max_nodes) max_nodes[i] = bt->groups[i].vmax;
        if (block) block[i] = bt->groups[i].block;
        if (grid) grid[i] = bt->groups[i].grid;
    }
    *count = n;
    return BP_OK;
}

int bp_batch_get_block_threads(const bp_batch *bt, uint32_t *states, uint32_t *block, uint32_t *count) {
    if (!bt || !count) return set_error(BP_ERR_INVALID, "null argument");
    const uint32_t n = (uint32_t)bt->groups.size();
    for (uint32_t i = 0; i < n && i < *count; ++i) {
        if (states) states[i] = (uint32_t)bt->groups[i].S;
        if (block) block[i] = bt->groups[i].block;
    }
    *count = n;
    return BP_OK;
}

int bp_batch_loopy(bp_batch *bt, const bp_batch_options *o, bp_batch_result *r) {
    NvtxRange nvtx("bp_batch_loopy");
    if (!bt || !o) return set_error(BP_ERR_INVALID, "null argument");
    if (o->delta_mode < BP_DELTA_AUTO || o->delta_mode > BP_DELTA_F64)
        return set_error(BP_ERR_INVALID, "unknown delta mode %d", o->delta_mode);
    const int serial = o->delta_mode == BP_DELTA_SERIAL_F32;
    if (serial && !bt->absdiff) {
        BP_CUDA(cudaMalloc((void **)&bt->absdiff, sizeof(float) * 2 * (bt->totMsgF + 4)));
        if (bt->exec) {
            cudaGraphExecDestroy(bt->exec);
            bt->exec = nullptr;
        }
    }
    if (o->block_threads) {
        if (o->block_threads % 32 || o->block_threads > 1024)
            return set_error(BP_ERR_INVALID, "block_threads must be a multiple of 32, at most 1024");
        for (auto &gr : bt->groups)
            if (gr.block != o->block_threads) {
                gr.block = o->block_threads;
                gr.grid = grid_for_group(bt, gr, gr.block);
                if (bt->exec) {
                    cudaGraphExecDestroy(bt->exec);
                    bt->exec = nullptr;
                }
            }
    }
    if (o->max_iterations == 0) return set_error(BP_ERR_INVALID, "max_iterations must be at least 1");
    // one CUDA graph per (options, tiling): the queue reset and every group's launch
    uint64_t key = (uint64_t)o->max_iterations | ((uint64_t)serial << 32) | ((uint64_t)(o->init_messages != 0) << 33);
    uint32_t tb;
    memcpy(&tb, &o->tolerance, 4);
    key ^= (uint64_t)tb << 34;
    for (auto &gr : bt->groups) key = key * 1000003ull + gr.block;
    if (!bt->exec || bt->exec_key != key) {
        if (bt->exec) {
            cudaGraphExecDestroy(bt->exec);
            bt->exec = nullptr;
        }
        const BatchArgs a = batch_args(bt, o->tolerance, o->max_iterations, serial, o->init_messages);
        cudaGraph_t graph = nullptr;
        BP_CUDA(cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeThreadLocal));
        int st = enqueue_batch(bt, a);
        cudaError_t ce = cudaStreamEndCapture(bt->stream, &graph);
        if (st) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
        cudaError_t ie = cudaGraphInstantiate(&bt->exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
        bt->exec_key = key;
    }
    BP_CUDA(cudaEventRecord(bt->ev0, bt->stream));
    BP_CUDA(cudaGraphLaunch(bt->exec, bt->stream));
    BP_CUDA(cudaEventRecord(bt->ev1, bt->stream));
    BP_CUDA(cudaEventSynchronize(bt->ev1));
    if (r) {
        std::vector<NetResult> res(bt->N);
        BP_CUDA(cudaMemcpyAsync(res.data(), bt->res, sizeof(NetResult) * bt->N, cudaMemcpyDeviceToHost, bt->stream));
        BP_CUDA(cudaStreamSynchronize(bt->stream));
        r->num_networks = bt->N;
        r->converged = 0;
        r->max_executed = 0;
        for (auto &x : res) {
            r->converged += x.converged;
            r->max_executed = std::max(r->max_executed, x.executed);
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, bt->ev0, bt->ev1);
        r->elapsed_ms = ms;
    }
    return BP_OK;
}

int bp_batch_network_results(bp_batch *bt, uint32_t *iterations, uint32_t *executed, int32_t *converged,
                             float *delta) {
    if (!bt) return set_error(BP_ERR_INVALID, "null batch");
    std::vector<NetResult> res(bt->N);
    BP_CUDA(cudaMemcpyAsync(res.data(), bt->res, sizeof(NetResult) * bt->N, cudaMemcpyDeviceToHost, bt->stream));
    BP_CUDA(cudaStreamSynchronize(bt->stream));
    for (uint32_t n = 0; n < bt->N; ++n) {
        if (iterations) iterations[n] = res[n].iterations;
        if (executed) executed[n] = res[n].executed;
        if (converged) converged[n] = (int32_t)res[n].converged;
        if (delta) delta[n] = res[n].delta;
    }
    return BP_OK;
}

}  // extern "C"
