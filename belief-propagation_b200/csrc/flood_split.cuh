// flood_split.cuh -- the split flooding schedule: one reference iteration as
// a send pass over the edges in source-range order followed by a node pass.
// Included by loopy.cu (it uses the control-block and delta machinery there).
//
// Why.  In k_flood the one random access is the gather Q[src] of the send
// buffer.  On a graph whose send buffers do not fit L2 (16.8M nodes x 2
// states = 134 MB), each 8-byte gather costs a 32-byte DRAM sector, about
// 1.4 GB of excess per iteration on the 67M-edge graph.  Here the edges are
// laid out a second time in "send order": grouped by the range of their
// source node (range_nodes consecutive ids, default 32 MB of send buffers per
// range) and in position order inside a range (engine.cu, split_build).
//
//   send pass (k_flood_send, edge-parallel over send order):
//       m_t = normalise(J . Q_t[src]), |m_{t-1} - m_t| into the delta,
//       m_t stored in send order.  Source ids, tables and old messages are
//       contiguous streams; the grid walks send order front to back (round r
//       of every block covers one window of it), so at any time the gathers
//       hit one range whose send buffers stay in L2.
//   node pass (k_flood_nodes, a thread per node):
//       each in-edge's message is read from send order through s_inv (the
//       send index of position p), in position order, so the product is
//       k_flood's phase 2 exactly; the node writes b_t and Q_{t+1}.  A node
//       tile's messages sit in a few contiguous runs of send order (one per
//       range), so these reads share sectors.  The last block to finish sums
//       the send pass's delta partials in a fixed order and applies the
//       stopping rule.
//
// Every fp32 operation is k_flood's, on the same operands in the same order
// (the product order inside a node is the position order), so beliefs and
// messages are bit-identical to k_flood's and the reference's.
//
// HBM bytes per iteration (S states): send pass 4S^2 + 4 + 4S + 4S per edge
// plus the gathers (about one sector per 4 nodes per range), node pass
// 4S + 4 per edge and 4 + 4S + 4S + 4S per node.  For S = 2: 48 B/edge +
// 28 B/node + ~V*8 of gathers, against k_flood's 44 B/edge + 28 B/node whose
// gathers cost a 32-byte sector each.
//
// A first form staged the send pass's streams through shared memory with
// bulk copies and scattered the messages into node tiles in shared memory;
// both kernels were latency-bound at low occupancy (2 CTAs of 8 warps per SM,
// short-scoreboard stalls; 1.18 ms per iteration against k_flood's 0.87 ms
// on the 16.8M-node graph), so both are now plain loads at full occupancy.
#pragma once

struct SplitArgs {
    uint32_t V, E;
    const uint32_t *in_ptr, *s_src, *s_edge, *s_inv;
    const float *s_joint;
    float *s_msg0, *s_msg1, *q0, *q1, *belief;
    double *partials;
    uint32_t nparts;
    float *absdiff;
    LoopyCtl *ctl;
};

constexpr int kSendThreads = 256;
constexpr int kNodeThreads = 256;
// resident blocks per SM the send pass's registers are capped for (48 warps,
// as k_flood's 1-2 state kernel)
template <int MS> constexpr int send_min_blocks() { return MS <= 2 ? 6 : 4; }

// Edges are assigned round by round: round r of block b covers send indices
// [(r * G + b) * NT, ... + NT), G = gridDim.x, so the whole grid moves
// through send order together.  One edge per thread per round; the next
// round's source id is loaded one round ahead (the load chain is then the
// gather alone).
template <int MS, bool SER>
__global__ void __launch_bounds__(kSendThreads, send_min_blocks<MS>()) k_flood_send(const SplitArgs a) {
    constexpr uint32_t NT = kSendThreads;
    __shared__ double red[NT / 32];
    LoopyCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint32_t it = ctl->it, ce = ctl->check_every;
    const bool want = (ce <= 1) || ((it + 1) % ce == 0);
    const int mp = (int)((ctl->msg_parity0 + it) & 1u), qp = (int)((ctl->q_parity0 + it) & 1u);
    const float *__restrict__ m_old = mp ? a.s_msg1 : a.s_msg0;
    float *__restrict__ m_new = mp ? a.s_msg0 : a.s_msg1;
    const float *__restrict__ q_in = qp ? a.q1 : a.q0;
    float *absd = SER ? check_buffer(ctl, a.absdiff, it, want) : nullptr;
    const uint64_t step = (uint64_t)gridDim.x * NT;
    double dsum = 0.0;
    uint64_t k = (uint64_t)blockIdx.x * NT + threadIdx.x;
    uint32_t s_cur = k < a.E ? __ldcs(a.s_src + k) : 0u;
    for (; k < a.E; k += step) {
        const uint64_t kn = k + step;
        const uint32_t s_nxt = kn < a.E ? __ldcs(a.s_src + kn) : 0u;
        float q[MS], jt[MS * MS], m[MS], o[MS];
        ldv<MS>(q_in + (size_t)s_cur * MS, q);
        ldv<MS * MS, kStream>(a.s_joint + k * (MS * MS), jt);
        if (want) ldv<MS, kStream>(m_old + k * MS, o);
        send_msg_regs<MS, true>(jt, q, MS, MS, m);
        if (want) {
            float ad[MS];
#pragma unroll
            for (int kk = 0; kk < MS; ++kk) {
                float d = FSUB(o[kk], m[kk]);
                if (d != d) d = 0.0f;
                d = fabsf(d);
                ad[kk] = d;
                dsum += (double)d;
            }
            if (SER && absd) stv<MS>(absd + (size_t)__ldg(a.s_edge + k) * MS, ad);
        }
        stv<MS, kStream>(m_new + k * MS, m);
        s_cur = s_nxt;
    }
    const double t = block_sum<NT>(dsum, red);
    if (threadIdx.x == 0) a.partials[blockIdx.x] = t;
}

// the last node-pass block to finish: the send pass's delta partials summed
// in a fixed order, then the stopping rule (serial mode: decided from the
// f64 sum and the serial sum's bounds, as k_flood's last block does)
template <int NT, bool SER>
__device__ __forceinline__ void split_finalize(const SplitArgs &a, bool want, double *red, bool *s_last, float *buf,
                                               uint32_t cap) {
    LoopyCtl *ctl = a.ctl;
    if (threadIdx.x == 0) {
        unsigned ticket;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(ticket) : "l"(&ctl->counter) : "memory");
        *s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!*s_last) return;
    __threadfence();
    double acc = 0.0;
    for (uint32_t k = threadIdx.x; k < a.nparts; k += NT) acc += __ldcg(a.partials + k);
    const double tot = block_sum<NT>(acc, red);
    if constexpr (SER) {
        finalize_serial<NT>(ctl, want, tot, a.absdiff, buf, cap);
        if (threadIdx.x == 0) ctl->counter = 0;
    } else if (threadIdx.x == 0) {
        ctl->counter = 0;
        finalize(ctl, want, (float)tot, tot);
    }
}

// marginalise (graph.c:1003-1023), then the next send buffer
// (graph.c:850-882) from the same messages: k_flood's phase 2, a thread per
// node, the messages read from send order through s_inv in position order
// (the second pass re-reads them, from L1).  Nodes grid-stride.  NV selects
// the form of the loads (sweeps; the same results): 0 plain, 1 the loop
// unrolled by 4 by the compiler, 2 the send indices and messages through
// the read-only path, 3 as 1 with the next node's row pointers and belief
// loaded one round ahead.  Measured forms that were slower, on the 16.8M-node
// graph with nodes renumbered by out-degree (ties by id): four messages
// loaded before their use (0.43 ms against 0.34 ms per launch), warp tiles
// staging a tile's messages through shared memory (0.45 ms), and a group of
// 4 lanes per node (1.6 ms).  With ties broken by in-degree, so that a warp's
// nodes have in-edge lists of similar length, this form takes 0.26 ms.
template <int MS, int NV>
__device__ __forceinline__ void node_msg(const SplitArgs &a, const float *__restrict__ m_new, uint32_t p, float *mm) {
    if constexpr (NV == 2) ldv<MS, kReadOnly>(m_new + (size_t)__ldg(a.s_inv + p) * MS, mm);
    else ldv<MS>(m_new + (size_t)a.s_inv[p] * MS, mm);
}

template <int MS, bool SER, int NV = 0>
__global__ void __launch_bounds__(kNodeThreads) k_flood_nodes(const SplitArgs a) {
    constexpr int NT = kNodeThreads;
    constexpr uint32_t CAP = SER ? 8u * NT : 1u;   // staging of the serial sum (serial mode only)
    __shared__ double red[NT / 32];
    __shared__ bool s_last;
    __shared__ __align__(16) float sbuf[CAP];
    LoopyCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint32_t it = ctl->it, ce = ctl->check_every;
    const bool want = (ce <= 1) || ((it + 1) % ce == 0);
    const int mp = (int)((ctl->msg_parity0 + it) & 1u), qp = (int)((ctl->q_parity0 + it) & 1u);
    const float *__restrict__ m_new = mp ? a.s_msg0 : a.s_msg1;
    float *__restrict__ q_out = qp ? a.q0 : a.q1;
    // NV 3: the next node's row pointers and belief are loaded one round
    // ahead, so a node's chain starts at its in-edges' send indices
    const uint32_t stride = gridDim.x * NT;
    uint32_t v = blockIdx.x * NT + threadIdx.x;
    uint32_t nr0 = 0, nr1 = 0;
    float nb[MS];
    if (NV == 3 && v < a.V) {
        nr0 = a.in_ptr[v];
        nr1 = a.in_ptr[v + 1];
        ldv<MS, kStream>(a.belief + (size_t)v * MS, nb);
    }
    for (; v < a.V; v += stride) {
        uint32_t r0, r1;
        float b[MS], prod[MS];
        if constexpr (NV == 3) {
            r0 = nr0;
            r1 = nr1;
#pragma unroll
            for (int s = 0; s < MS; ++s) b[s] = nb[s];
            const uint64_t vn = (uint64_t)v + stride;
            if (vn < a.V) {
                nr0 = a.in_ptr[vn];
                nr1 = a.in_ptr[vn + 1];
                ldv<MS, kStream>(a.belief + (size_t)vn * MS, nb);
            }
        } else {
            r0 = a.in_ptr[v];
            r1 = a.in_ptr[v + 1];
            ldv<MS, kStream>(a.belief + (size_t)v * MS, b);
        }
#pragma unroll
        for (int s = 0; s < MS; ++s) prod[s] = 1.0f;
        if constexpr (NV == 1 || NV == 3) {
#pragma unroll 4
            for (uint32_t p = r0; p < r1; ++p) {
                float mm[MS];
                node_msg<MS, NV>(a, m_new, p, mm);
                combine<MS, true>(prod, mm, MS);
            }
        } else {
            for (uint32_t p = r0; p < r1; ++p) {
                float mm[MS];
                node_msg<MS, NV>(a, m_new, p, mm);
                combine<MS, true>(prod, mm, MS);
            }
        }
        if (r1 > r0) {
#pragma unroll
            for (int s = 0; s < MS; ++s) b[s] = FMUL(b[s], prod[s]);
        }
        normalise<MS, true>(b, MS);
        stv<MS, kStream>(a.belief + (size_t)v * MS, b);
        float qo[MS];
#pragma unroll
        for (int s = 0; s < MS; ++s) qo[s] = b[s];
        for (uint32_t p = r0; p < r1; ++p) {
            float mm[MS];
            node_msg<MS, NV>(a, m_new, p, mm);
            combine<MS, true>(qo, mm, MS);
        }
        stv<MS>(q_out + (size_t)v * MS, qo);
    }
    split_finalize<NT, SER>(a, want, red, &s_last, sbuf, CAP);
}

// the latest messages into send order before the loop, and both message
// arrays back to position order after it
template <int MS>
__global__ void k_to_send_order(const uint32_t *__restrict__ s_pos, uint32_t E, const float *__restrict__ m_pos,
                                float *__restrict__ m_send) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= E) return;
    float m[MS];
    ldv<MS>(m_pos + (size_t)s_pos[k] * MS, m);
    stv<MS>(m_send + k * MS, m);
}

template <int MS>
__global__ void k_from_send_order(const uint32_t *__restrict__ s_pos, uint32_t E, const float *__restrict__ m_send,
                                  float *__restrict__ m_pos) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= E) return;
    float m[MS];
    ldv<MS>(m_send + k * MS, m);
    stv<MS>(m_pos + (size_t)s_pos[k] * MS, m);
}
