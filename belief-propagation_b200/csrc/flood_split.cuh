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
//       contiguous streams, moved into a ring of shared-memory stages by
//       bulk asynchronous copies (cp.async.bulk, no multicast, evict-first);
//       the blocks walk the chunks in order, so at any time the grid gathers
//       from one range whose send buffers stay in L2.
//   node pass (k_flood_nodes, node tiles of 128 nodes):
//       the tile's messages are one contiguous segment per range of the send
//       order (segment table `seg`); each message goes to shared memory at
//       its position offset (s_off), then each node multiplies its in-edges'
//       messages in position order exactly as k_flood's phase 2 does, writes
//       b_t and Q_{t+1}.  The last block to finish sums the send pass's delta
//       partials in a fixed order and applies the stopping rule.
//
// Every fp32 operation is k_flood's, on the same operands in the same order
// (the product order inside a node is the position order), so beliefs and
// messages are bit-identical to k_flood's and the reference's.
//
// HBM bytes per iteration (S states): send pass 4S^2 + 4 + 4S + 4S per edge
// plus the gathers (about one sector per 4 nodes per range), node pass
// 4S + 2 per edge and 4 + 4S + 4S + 4S per node.  For S = 2: 46 B/edge +
// 28 B/node + ~V*8 of gathers, against k_flood's 44 B/edge + 28 B/node whose
// gathers cost a sector each.
#pragma once

struct SplitArgs {
    uint32_t V, E, nchunks, ntiles, R, nparts;
    const uint32_t *in_ptr, *s_src, *s_edge, *seg;
    const uint16_t *s_off;
    const float *s_joint;
    float *s_msg0, *s_msg1, *q0, *q1, *belief;
    double *partials;
    float *absdiff;
    LoopyCtl *ctl;
};

// send pass: CH edges per chunk, ST stages of (source ids, tables, old
// messages) per CTA of NT threads
template <int MS, uint32_t CH_, int ST_, uint32_t NT_>
struct SendCfgT {
    static constexpr uint32_t NT = NT_;
    static constexpr uint32_t CH = CH_;
    static constexpr uint32_t U = CH / NT;   // edges per thread per chunk
    static constexpr int ST = ST_;
    static constexpr uint32_t SRC = 0;
    static constexpr uint32_t JNT = SRC + CH * 4;
    static constexpr uint32_t MOLD = JNT + CH * MS * MS * 4;
    static constexpr uint32_t STAGE = round16(MOLD + CH * MS * 4);
    static constexpr uint32_t BAR = ST * STAGE;
    static constexpr uint32_t SMEM = BAR + 16 * ST;
    static_assert(MS >= 1 && MS <= 4, "split schedule: 1 to 4 states");
    static_assert(CH % NT == 0 && (CH * 4) % 16 == 0, "whole rounds, 16-byte aligned sections");
};
// the default shape: stages under 29 KB, three of them
template <int MS>
using SendCfg = SendCfgT<MS, (MS == 1 ? 2048u : (MS == 2 ? 1024u : (MS == 3 ? 512u : 256u))), 3, 256u>;

// node pass: tiles of NT nodes holding at most EB in-edges (8 in-edges per
// node on average with 1-2 states, 16 with 3-4: a tile's messages take 8 or
// 32 KB of shared memory per 128 nodes)
template <int MS, uint32_t NT_ = 128>
struct NodeCfg {
    static constexpr uint32_t NT = NT_;
    static constexpr uint32_t EB = (MS <= 2 ? 2048u : 8192u) / MS * (NT_ / 128u);
    static constexpr uint32_t RMAX = 32;   // source ranges at most
};

__device__ __forceinline__ uint64_t l2_evict_first_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// bulk copy global -> shared with an L2 eviction-priority policy
__device__ __forceinline__ void bulk_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], "
        "%4;" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
        : "memory");
}

// issue chunk c into stage `st` (one thread).  Chunk starts are multiples of
// CH, so every source address is 16-byte aligned; lengths are rounded up to
// 16 bytes and the send-order arrays carry padding past their ends.  The
// mbarrier expects exactly the bytes issued.
template <int MS, typename C>
__device__ void send_issue(const SplitArgs &a, const float *m_old, bool want, uint32_t c, unsigned char *st,
                           uint64_t *bar, uint64_t pol) {
    const uint32_t k0 = c * C::CH, n = min(C::CH, a.E - k0);
    const uint32_t b_src = round16(n * 4), b_j = round16(n * MS * MS * 4), b_m = want ? round16(n * MS * 4) : 0u;
    mbar_arrive_expect_tx(bar, b_src + b_j + b_m);
    bulk_g2s_hint(st + C::SRC, a.s_src + k0, b_src, bar, pol);
    bulk_g2s_hint(st + C::JNT, a.s_joint + (size_t)k0 * (MS * MS), b_j, bar, pol);
    if (b_m) bulk_g2s_hint(st + C::MOLD, m_old + (size_t)k0 * MS, b_m, bar, pol);
}

// the gathers Q_t[src] of chunk c's edges (thread's U edges) into registers
template <int MS, typename C>
__device__ __forceinline__ void send_gather(const SplitArgs &a, const unsigned char *st, uint32_t c,
                                            const float *__restrict__ q_in, float (*q)[MS]) {
    const uint32_t k0 = c * C::CH, n = min(C::CH, a.E - k0);
    const uint32_t *src_s = reinterpret_cast<const uint32_t *>(st + C::SRC);
#pragma unroll
    for (uint32_t u = 0; u < C::U; ++u) {
        const uint32_t j = threadIdx.x + u * C::NT;
        if (j < n) ldv<MS>(q_in + (size_t)src_s[j] * MS, q[u]);
    }
}

// The chunks of a CTA form a pipeline: chunk i+ST-1's bulk copies are in
// flight, chunk i+1's gathers are in flight (issued from its landed source
// ids), and chunk i is computed from its stage and its gathered values.
template <int MS, bool SER, typename C>
__global__ void __launch_bounds__(C::NT) k_flood_send(const SplitArgs a) {
    constexpr uint32_t NT = C::NT;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double red[NT / 32];
    __shared__ uint32_t s_err;

    LoopyCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint32_t it = ctl->it, ce = ctl->check_every;
    const bool want = (ce <= 1) || ((it + 1) % ce == 0);
    const int mp = (int)((ctl->msg_parity0 + it) & 1u), qp = (int)((ctl->q_parity0 + it) & 1u);
    const float *__restrict__ m_old = mp ? a.s_msg1 : a.s_msg0;
    float *__restrict__ m_new = mp ? a.s_msg0 : a.s_msg1;
    const float *__restrict__ q_in = qp ? a.q1 : a.q0;
    float *absd = SER ? check_buffer(ctl, a.absdiff, it, want) : nullptr;
    const uint64_t pol = l2_evict_first_policy();
    const uint32_t tid = threadIdx.x;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + C::BAR);

    if (tid == 0) {
        s_err = 0;
        for (int i = 0; i < C::ST; ++i) mbar_init(bars + i, 1);
        fence_mbar_init();
        for (int i = 0; i < C::ST; ++i) {
            const uint32_t c = blockIdx.x + (uint32_t)i * gridDim.x;
            if (c < a.nchunks) send_issue<MS, C>(a, m_old, want, c, smem + i * C::STAGE, bars + i, pol);
        }
    }
    __syncthreads();

    // stage of chunk number i of this CTA landed: every thread may read it
    auto wait_stage = [&](uint32_t i) -> bool {
        const int si = (int)(i % C::ST);
        const uint32_t par = (i / C::ST) & 1u;
        if (tid == 0 && !mbar_wait_bounded(bars + si, par, kWaitNs)) s_err = 1;
        __syncthreads();
        if (s_err) return false;
        mbar_try_wait(bars + si, par);   // completed: orders this thread's reads after the copies
        return true;
    };

    double dsum = 0.0;
    float q[C::U][MS], qn[C::U][MS];
    uint32_t i = 0;
    bool ok = blockIdx.x >= a.nchunks || wait_stage(0);
    if (ok && blockIdx.x < a.nchunks) send_gather<MS, C>(a, smem, blockIdx.x, q_in, qn);
    for (uint32_t c = blockIdx.x; ok && c < a.nchunks; c += gridDim.x, ++i) {
#pragma unroll
        for (uint32_t u = 0; u < C::U; ++u)
#pragma unroll
            for (int s = 0; s < MS; ++s) q[u][s] = qn[u][s];
        const uint32_t cn = c + gridDim.x;
        if (cn < a.nchunks) {
            if (!wait_stage(i + 1)) {
                ok = false;
                break;
            }
            send_gather<MS, C>(a, smem + ((i + 1) % C::ST) * C::STAGE, cn, q_in, qn);
        }
        unsigned char *st = smem + (i % C::ST) * C::STAGE;
        const uint32_t k0 = c * C::CH, n = min(C::CH, a.E - k0);
        const float *j_s = reinterpret_cast<const float *>(st + C::JNT);
        const float *mo_s = reinterpret_cast<const float *>(st + C::MOLD);
#pragma unroll
        for (uint32_t u = 0; u < C::U; ++u) {
            const uint32_t j = tid + u * NT;
            if (j < n) {
                float jt[MS * MS], m[MS];
                ldv<MS * MS>(j_s + (size_t)j * (MS * MS), jt);
                send_msg_regs<MS, true>(jt, q[u], MS, MS, m);
                if (want) {
                    float o[MS], ad[MS];
                    ldv<MS>(mo_s + (size_t)j * MS, o);
#pragma unroll
                    for (int kk = 0; kk < MS; ++kk) {
                        float d = FSUB(o[kk], m[kk]);
                        if (d != d) d = 0.0f;
                        d = fabsf(d);
                        ad[kk] = d;
                        dsum += (double)d;
                    }
                    if (SER && absd) stv<MS>(absd + (size_t)__ldg(a.s_edge + k0 + j) * MS, ad);
                }
                stv<MS, kStream>(m_new + (size_t)(k0 + j) * MS, m);
            }
        }
        // every thread is done with the stage; it takes the chunk ST ahead
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            const uint32_t nc = c + (uint32_t)C::ST * gridDim.x;
            if (nc < a.nchunks) send_issue<MS, C>(a, m_old, want, nc, st, bars + (i % C::ST), pol);
        }
    }

    if (!ok) {
        // a stage never completed: report it, wait (bounded) for the copies
        // still in flight into this CTA's stages, and leave
        if (tid == 0) {
            atomicExch(&ctl->done, 3u);
            for (uint32_t j = 0; j < (uint32_t)C::ST; ++j) {
                const uint32_t kk = i + j, c = blockIdx.x + kk * gridDim.x;
                if (c < a.nchunks) mbar_wait_bounded(bars + (kk % C::ST), (kk / C::ST) & 1u, kWaitNs);
            }
        }
        return;
    }
    const double t = block_sum<NT>(dsum, red);
    if (tid == 0) a.partials[blockIdx.x] = t;
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

template <int MS, bool SER, typename C>
__global__ void __launch_bounds__(C::NT) k_flood_nodes(const SplitArgs a) {
    constexpr uint32_t NT = C::NT;
    constexpr uint32_t UB = 4;   // messages per thread in flight while they go to shared memory
    __shared__ __align__(16) float sm[C::EB * MS];
    __shared__ uint32_t s_beg[C::RMAX], s_pre[C::RMAX + 1];
    __shared__ double red[NT / 32];
    __shared__ bool s_last;

    LoopyCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint32_t it = ctl->it, ce = ctl->check_every;
    const bool want = (ce <= 1) || ((it + 1) % ce == 0);
    const int mp = (int)((ctl->msg_parity0 + it) & 1u), qp = (int)((ctl->q_parity0 + it) & 1u);
    const float *__restrict__ m_new = mp ? a.s_msg0 : a.s_msg1;
    float *__restrict__ q_out = qp ? a.q0 : a.q1;
    const uint32_t tid = threadIdx.x, R = a.R;

    for (uint32_t tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x) {
        const uint32_t v0 = tile * NT, v = v0 + tid;
        const bool has = v < a.V;
        const uint32_t e0 = a.in_ptr[v0];
        uint32_t r0 = 0, r1 = 0;
        float b[MS];
        if (has) {
            r0 = a.in_ptr[v];
            r1 = a.in_ptr[v + 1];
            ldv<MS, kStream>(a.belief + (size_t)v * MS, b);
        }
        // this tile's segment of each range
        if (tid < R) {
            const uint32_t b0 = a.seg[(size_t)tid * a.ntiles + tile], b1 = a.seg[(size_t)tid * a.ntiles + tile + 1];
            s_beg[tid] = b0;
            s_pre[tid + 1] = b1 - b0;
        }
        __syncthreads();
        if (tid == 0) {
            s_pre[0] = 0;
            for (uint32_t r = 0; r < R; ++r) s_pre[r + 1] += s_pre[r];
        }
        __syncthreads();
        const uint32_t total = s_pre[R];
        // messages back to position order in shared memory: UB of them
        // per thread loaded before the first is stored
        for (uint32_t j0 = tid; j0 < total; j0 += NT * UB) {
            float m[UB][MS];
            uint32_t o[UB];
#pragma unroll
            for (uint32_t u = 0; u < UB; ++u) {
                const uint32_t j = j0 + u * NT;
                if (j < total) {
                    uint32_t r = 0;
                    while (j >= s_pre[r + 1]) ++r;
                    const size_t k = (size_t)s_beg[r] + (j - s_pre[r]);
                    ldv<MS, kStream>(m_new + k * MS, m[u]);
                    o[u] = __ldcs(a.s_off + k);
                }
            }
#pragma unroll
            for (uint32_t u = 0; u < UB; ++u)
                if (j0 + u * NT < total) stv<MS>(sm + (size_t)o[u] * MS, m[u]);
        }
        __syncthreads();
        // marginalise (graph.c:1003-1023), then the next send buffer
        // (graph.c:850-882) from the same messages: k_flood's phase 2
        if (has) {
            float prod[MS];
#pragma unroll
            for (int s = 0; s < MS; ++s) prod[s] = 1.0f;
            for (uint32_t p = r0; p < r1; ++p) {
                float mm[MS];
                ldv<MS>(sm + (size_t)(p - e0) * MS, mm);
                combine<MS, true>(prod, mm, MS);
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
                ldv<MS>(sm + (size_t)(p - e0) * MS, mm);
                combine<MS, true>(qo, mm, MS);
            }
            stv<MS>(q_out + (size_t)v * MS, qo);
        }
        __syncthreads();   // shared memory is free for the next tile
    }
    split_finalize<NT, SER>(a, want, red, &s_last, sm, C::EB * MS);
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
