// loopy.cu -- synchronous flooding BP on the destination-sorted layout.
//
// One reference iteration (loopy_propagate_one_iteration, graph.c:1121-1183,
// then the delta of loopy_propagate_until, graph.c:1294-1310) is ONE launch of
// k_flood here.  The reference computes, per iteration t,
//     Q_t(v)  = b_{t-1}(v) * prod_{in-edges, order} m_{t-1}        (send buffer)
//     m_t(e)  = normalise(J_e . Q_t(src e))                          (send)
//     b_t(v)  = normalise(b_{t-1}(v) * prod_{in-edges} m_t)          (marginalise)
// and Q_{t+1}(v) is b_t(v) times the same incoming m_t, so the node step of
// iteration t can emit Q_{t+1} while the messages are still on chip.  k_flood
// therefore computes, for a tile of consecutive destination nodes:
//   phase 1 (edge-parallel over the tile's in-edges, contiguous in HBM):
//       m_t = normalise(J . Q_t[src]), |m_{t-1} - m_t| into the delta,
//       m_t to HBM and to shared memory;
//   phase 2 (node-parallel): P = prod m_t, b_t = normalise(b_{t-1} * P),
//       Q_{t+1} = b_t * prod m_t (from shared memory);
// and the last block to finish reduces the delta and applies the stopping
// rule, so the loop runs as a CUDA graph without host round trips.  Each value
// goes through the same fp32 operations in the same order as the reference.
//
// HBM bytes per iteration (S states, fp32, u32 indices): per edge
// 4S^2 (J) + 4 (src) + 4S (Q[src] gather) + 4S (old m) + 4S (new m), per node
// 4 (row ptr) + 4S (b read) + 4S (b write) + 4S (Q write) + 4S (Q read is
// counted per edge).  For S = 2: 44 B/edge + 28 B/node.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "bp_device.cuh"
#include "bp_serial.cuh"
#include "bp_internal.h"

namespace bpx {

// nodes per tile (= threads per block) and the shared-memory message buffer;
// with 1-2 states 128-node tiles (12 blocks per SM) measured 2 % faster than
// 256-node tiles on the 16M-node graph, 512-node tiles 4 % slower
template <int MS> constexpr int flood_nt() { return MS <= 2 ? 128 : (MS <= 4 ? 256 : 128); }
template <int MS> constexpr int flood_smem_floats() { return MS <= 2 ? 2048 : 8192; }
// in-edges per thread per phase-1 round of k_flood (tables held in registers)
template <int MS> constexpr int flood_unroll() { return MS <= 2 ? 1 : (MS <= 4 ? 2 : 1); }
// resident blocks per SM the register allocation must allow.  With 1-2
// states, 48 warps of one edge per thread at 40 registers measured fastest on
// the 16M-node graph: 0.93 ms against 1.07 ms for 32 warps of 4 edges per
// thread at 64 registers; more warps hide the gather better than more
// gathers per warp.
template <int MS, int FU> constexpr int flood_min_blocks() { return MS <= 2 ? (FU >= 4 ? 8 : 12) : 1; }

struct FloodArgs {
    uint32_t V;          // tiles cover nodes [v_base, V)
    uint32_t v_base;     // first node of tile 0 (a node range of a sharded run; else 0)
    // send-buffer entries of nodes below this id are gathered and written
    // with an L2 evict-last policy (renumbered graphs: the nodes with the
    // most out-edges, i.e. the most re-read entries); 0 = none
    uint32_t hot;
    // one in-edge per thread: 1 = the next round's source id is loaded one
    // round ahead, 2 = its table and old message too
    uint32_t pipe;
    const uint32_t *in_ptr, *in_src, *pos_edge;
    const uint8_t *node_s, *pos_dims;
    const float *joint;
    float *belief;
    float *msg0, *msg1, *q0, *q1;
    double *partials;
    float *absdiff;
    LoopyCtl *ctl;
};

// the previous check's delta takes the current one's value and bounds
__device__ __forceinline__ void keep_prev(LoopyCtl *c, float df, double dd) {
    c->prev_f = df;
    c->prev_d = dd;
    c->plo = c->dlo;
    c->phi = c->dhi;
    c->prev_exact = c->delta_exact;
    c->prev_ref = c->delta_ref;
    c->prev_buf = c->cur_buf;
}

// the reference's loop bookkeeping (graph.c:1313-1318; _acc: :1410-1414)
// once the stopping rule's outcome `stop` is known; one thread
__device__ void finalize_with(LoopyCtl *c, bool has_delta, bool stop, float df, double dd) {
    const uint32_t it = c->it, ce = c->check_every, max_it = c->max_it;
    if (has_delta) {
        c->delta_f = df;
        c->delta_d = dd;
    }
    if (ce <= 1) {
        if (stop) {
            c->done = 1;
            c->ret = it;
            c->final_i = it;
        } else {
            if (it < max_it - 1) keep_prev(c, df, dd);
            if (it + 1 >= max_it) {
                c->done = 2;
                c->ret = max_it;
                c->final_i = max_it;
            }
        }
    } else if (has_delta) {
        const uint32_t i_ref = it + 1 - ce;
        if (stop) {
            c->done = 1;
            c->ret = c->num_iter;
            c->final_i = i_ref;
        } else {
            keep_prev(c, df, dd);
            c->num_iter += ce;
            if (i_ref + ce >= max_it) {
                c->done = 2;
                c->ret = c->num_iter;
                c->final_i = i_ref + ce;
            }
        }
    }
    c->it = it + 1;
}

// the f64 delta's stopping rule (the reference's, on the f64 sum); one thread
__device__ void finalize(LoopyCtl *c, bool has_delta, float df, double dd) {
    const bool stop = has_delta && ((dd < (double)c->tol) || (fabs(dd - c->prev_d) < (double)c->tol));
    finalize_with(c, has_delta, stop, df, dd);
}

// ---- the reference's serial fp32 delta, decided from bounds -------------
//
// The reference sums the n = E * stride terms t_i = |m_old - m_new| >= 0 in
// fp32, one add after another in edge-id order (graph.c:1300-1309), and
// stops when  delta < tol  or  |delta - previous_delta| < tol  (:1313).
// Each of the n - 1 rounded adds errs by at most u = 2^-24 (+ 2^-52 for the
// reference's add through double) of its exact result, which is at most
// (1 + gamma) S, S = sum t_i; so the serial sum s lies within
// gamma_(n-1) = (n-1)u / (1 - (n-1)u) of S (Higham, Accuracy and Stability of
// Numerical Algorithms, 2nd ed., section 4.2), plus 2^-149 per add for a
// subnormal result.  S itself comes from the iteration kernel's f64 sum of
// the same floats, within 2^-20 relative for n < 2^22.  With directed
// rounding these give an interval [lo, hi] that contains s.  When the
// intervals of s and of the previous check's delta decide both comparisons,
// the outcome is the reference's without forming s; otherwise the serial
// sum is formed (the previous one too if its interval still straddles), and
// the decision is exact.  The iteration count, messages and beliefs are
// therefore the reference's in every case.

__device__ __forceinline__ uint32_t check_index(uint32_t it, uint32_t ce) { return ce <= 1 ? it : (it + 1) / ce - 1; }


// the reference's serial fp32 sum of x[0, n) in index order (graph.c:1300-1309)
// as one dependent chain of adds: thread 0 runs the chain out of shared
// memory while threads 32.. stage the next `ch` terms into the other half of
// buf (2 * ch floats, 16-byte aligned, ch % 4 == 0).  Every thread of the
// block calls it and gets the sum.  Kept as the plain form the parallel one
// below is checked against.
template <int NT>
__device__ float block_serial_sum_chain(const float *__restrict__ x, uint64_t n, float *buf, uint32_t ch) {
    static_assert(NT >= 64, "a staging warp besides the chain's");
    __shared__ float s_res;
    const uint64_t nch = (n + ch - 1) / ch;
    auto stage = [&](uint64_t c) {
        const uint64_t base = c * ch;
        const uint32_t cnt = (uint32_t)min((uint64_t)ch, n - base);
        float *dst = buf + (c & 1) * ch;
        for (uint32_t k = threadIdx.x - 32; k < cnt; k += NT - 32) dst[k] = __ldcg(x + base + k);
    };
    __syncthreads();   // buf is free
    if (threadIdx.x >= 32 && nch) stage(0);
    __syncthreads();
    float s = 0.0f;
    for (uint64_t c = 0; c < nch; ++c) {
        if (threadIdx.x >= 32) {
            if (c + 1 < nch) stage(c + 1);
        } else if (threadIdx.x == 0) {
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
    if (threadIdx.x == 0) s_res = s;
    __syncthreads();
    return s_res;
}

// ---- the same serial sum, formed in parallel -----------------------------
//
// For non-negative terms the running sum s never decreases.  While s stays
// in one binade [2^e, 2^(e+1)) -- subnormals: [0, 2^-126) -- the floats
// there are the multiples m U of one unit U, and rounding s + t to nearest
// moves s by t rounded to a multiple of U: by floor(t/U) or floor(t/U) + 1,
// the choice fixed by t alone except at an exact tie, where it goes to the
// even m and so depends on the parity of m.  Each term is therefore a map
// m -> m + c(m mod 2), a pair (c_even, c_odd); pairs compose associatively
// (the parity of m after the first map is that of its increment, plus one
// from an odd start), so a block scan of the pairs gives m before every
// term, exactly.  The binade holds while m + floor(t/U) < 2^24 (2^23 for
// subnormals; the sum may round up onto the binade's top, 2^(e+1), and the
// next term then leaves).  The first term that leaves the binade, or is inf,
// is added by one thread, and the scan resumes in the new binade: the sum
// crosses O(log(n)) binades.  The result is bit for bit the one-by-one sum.
struct SumStep {
    uint32_t e, o;   // increment of m from an even / odd m
};
constexpr uint32_t kSumSat = 1u << 30;   // saturation: above every binade top

__device__ __forceinline__ uint32_t sum_sat(uint32_t a, uint32_t b) { return min(a + b, kSumSat); }

// a, then b
__device__ __forceinline__ SumStep sum_compose(SumStep a, SumStep b) {
    SumStep c;
    c.e = sum_sat(a.e, (a.e & 1u) ? b.o : b.e);
    c.o = sum_sat(a.o, (a.o & 1u) ? b.e : b.o);
    return c;
}

// term t against the binade with unit 2^eu: fl = floor(t / U) (saturated),
// the step's pair, and whether t is inf or NaN (added one by one)
__device__ __forceinline__ SumStep sum_term(float t, int eu, uint32_t &fl, bool &special) {
    const uint32_t tb = __float_as_uint(t);
    const uint32_t Et = (tb >> 23) & 0xffu;
    special = Et == 0xffu;
    const uint32_t Mt = Et ? ((tb & 0x7fffffu) | 0x800000u) : (tb & 0x7fffffu);
    const int shift = (Et ? (int)Et - 150 : -149) - eu;
    SumStep st;
    if (Mt == 0u) {
        fl = 0u;
        st.e = st.o = 0u;
    } else if (shift >= 0) {
        fl = shift >= 7 ? kSumSat : min(Mt << shift, kSumSat);
        st.e = st.o = fl;
    } else if (shift <= -26) {   // t < U / 4
        fl = 0u;
        st.e = st.o = 0u;
    } else {
        const uint32_t sh = (uint32_t)(-shift);
        fl = Mt >> sh;
        const uint32_t rem = Mt & ((1u << sh) - 1u), half = 1u << (sh - 1u);
        if (rem == half) {   // tie: to the even m
            st.e = fl + (fl & 1u);
            st.o = fl + ((fl + 1u) & 1u);
        } else {
            st.e = st.o = fl + (rem > half ? 1u : 0u);
        }
    }
    return st;
}

__device__ __forceinline__ uint32_t sum_apply(uint32_t m, SumStep st) { return sum_sat(m, (m & 1u) ? st.o : st.e); }

// the reference's serial fp32 sum of x[0, n) (graph.c:1300-1309), exactly, for
// non-negative terms; every thread of the block calls it and gets the sum.
// buf: cap floats of shared memory, cap >= 3 * NT.
template <int NT>
__device__ float block_serial_sum(const float *__restrict__ x, uint64_t n, float *buf, uint32_t cap) {
    static_assert(NT % 32 == 0 && NT <= 1024, "whole warps");
    constexpr int NW = NT / 32;
    constexpr uint32_t kHead = 32;   // terms added one by one at the start
    __shared__ uint32_t s_we[NW], s_wo[NW];
    __shared__ uint32_t s_first, s_m;
    __shared__ float s_val;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, w = tid >> 5;
    uint32_t K = cap / NT;
    K = (K > 1u ? K - 1u : 1u) & ~1u;   // terms per thread; row stride K + 1 is odd
    K = min(max(K, 2u), 30u);
    const uint32_t KS = K + 1u, P = NT * K;
    float s = 0.0f;
    __syncthreads();   // buf is free
    for (uint64_t i = 0; i < n;) {
        const uint32_t cnt = (uint32_t)min((uint64_t)P, n - i);
        for (uint32_t k = tid; k < cnt; k += NT) buf[(k / K) * KS + k % K] = __ldcg(x + i + k);
        __syncthreads();
        uint32_t pos = 0;
        if (i == 0) {   // the start: the sum crosses binades every few terms
            if (tid == 0) {
                const uint32_t h = min(kHead, cnt);
                for (uint32_t k = 0; k < h; ++k) s = FADD(s, buf[(k / K) * KS + k % K]);
                s_val = s;
            }
            __syncthreads();
            s = s_val;
            pos = min(kHead, cnt);
        }
        while (pos < cnt) {
            const uint32_t sb = __float_as_uint(s);
            const uint32_t Es = sb >> 23;
            if (Es >= 0xffu) break;   // inf (or NaN): it stays
            const int eu = Es ? (int)Es - 150 : -149;
            const uint32_t m0 = Es ? ((sb & 0x7fffffu) | 0x800000u) : sb;
            const uint32_t top = Es ? 0x1000000u : 0x800000u;
            const uint32_t a0 = max(tid * K, pos), a1 = min(tid * K + K, cnt);
            const float *row = buf + tid * KS - tid * K;   // row[k] for k in [tid K, tid K + K)
            SumStep acc{0u, 0u};
            for (uint32_t k = a0; k < a1; ++k) {
                uint32_t fl;
                bool sp;
                acc = sum_compose(acc, sum_term(row[k], eu, fl, sp));
            }
            // block exclusive scan of the threads' maps
            SumStep inc = acc;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                SumStep o;
                o.e = __shfl_up_sync(0xffffffffu, inc.e, d);
                o.o = __shfl_up_sync(0xffffffffu, inc.o, d);
                if ((int)lane >= d) inc = sum_compose(o, inc);
            }
            if (lane == 31u) {
                s_we[w] = inc.e;
                s_wo[w] = inc.o;
            }
            if (tid == 0) s_first = cnt;
            __syncthreads();
            SumStep pre{0u, 0u};
            for (uint32_t ww = 0; ww < w; ++ww) pre = sum_compose(pre, SumStep{s_we[ww], s_wo[ww]});
            SumStep ex;
            ex.e = __shfl_up_sync(0xffffffffu, inc.e, 1);
            ex.o = __shfl_up_sync(0xffffffffu, inc.o, 1);
            if (lane == 0u) ex = SumStep{0u, 0u};
            pre = sum_compose(pre, ex);
            // m before each of this thread's terms; the first that leaves
            // the binade (or is inf) ends the run
            uint32_t m = sum_apply(m0, pre), bad = cnt;
            for (uint32_t k = a0; k < a1; ++k) {
                uint32_t fl;
                bool sp;
                const SumStep st = sum_term(row[k], eu, fl, sp);
                if (sp || sum_sat(m, fl) >= top) {
                    bad = k;
                    break;
                }
                m = sum_apply(m, st);
            }
            if (bad < cnt) atomicMin(&s_first, bad);
            __syncthreads();
            const uint32_t j = s_first;
            // m just before term j (after the last term when j == cnt)
            const uint32_t owner = (j < cnt ? j : cnt - 1u) / K;
            if (tid == owner) s_m = m;
            __syncthreads();
            if (tid == 0) {
                uint32_t mm = s_m;
                s = __uint_as_float((Es << 23) + mm - (Es ? 0x800000u : 0u));
                if (j < cnt) {
                    // the leaving term, then (when the run was short) a few
                    // more one by one
                    const uint32_t stop = (j - pos < 32u) ? min(cnt, j + 1u + 64u) : j + 1u;
                    for (uint32_t k = j; k < stop; ++k) s = FADD(s, buf[(k / K) * KS + k % K]);
                    s_first = stop;
                } else {
                    s_first = cnt;
                }
                s_val = s;
            }
            __syncthreads();
            s = s_val;
            pos = s_first;
            __syncthreads();   // s_first is rewritten next round
        }
        i += cnt;
        __syncthreads();   // buf is rewritten next pass
        if (__float_as_uint(s) >> 23 >= 0xffu) break;
    }
    return s;
}

// the serial sum by whichever form is faster for the block: the parallel
// scan needs at least 256 threads to beat the chain (measured on 80k terms:
// 1024 threads with 8192 floats of staging 140 us, 256 threads 180-190 us,
// the chain 224 us, 128 threads with 2048 floats 257 us)
template <int NT>
__device__ __forceinline__ float exact_serial_sum(const float *x, uint64_t n, float *buf, uint32_t cap) {
    if (NT >= 256 && cap >= 8u * NT) return block_serial_sum<NT>(x, n, buf, cap);
    return block_serial_sum_chain<NT>(x, n, buf, (cap / 2u) & ~3u);
}

// one serial-mode check: s (the reference's delta) in [lo, hi], the
// previous delta in [plo, phi], d = serial_decide's outcome
struct SerialCheck {
    double T, lo, hi, plo, phi;
    float s;   // (float)T until the serial sum is known
    bool s_exact, p_exact;
    bool s_ref, p_ref;   // narrowed from the terms' errors
    bool p_new;          // [plo, phi] changed in this check
    int d;
    uint32_t sums, refines, cb;
};

// the decision from the bounds alone; every thread, the same T
__device__ SerialCheck serial_check(const LoopyCtl *c, double T) {
    SerialCheck x;
    x.T = T;
    x.plo = c->plo;
    x.phi = c->phi;
    x.p_exact = c->prev_exact != 0;
    x.p_ref = c->prev_ref != 0;
    x.s_exact = x.s_ref = x.p_new = false;
    x.sums = x.refines = 0;
    x.cb = check_index(c->it, c->check_every) % 3u;
    x.s = (float)T;
    serial_interval(T, c->n_terms, x.lo, x.hi);
    x.d = serial_decide(x.lo, x.hi, false, x.plo, x.phi, x.p_exact, c->tol);
    return x;
}

// a narrowed interval [lo, hi] of s (which == 0) or of the previous delta
__device__ __forceinline__ void serial_narrow(SerialCheck &x, int which, double lo, double hi) {
    double &L = which ? x.plo : x.lo, &H = which ? x.phi : x.hi;
    L = fmax(L, lo);
    H = fmin(H, hi);
    float f;
    const bool pinned = interval_pins(L, H, f);
    if (pinned) L = H = (double)f;
    if (which) {
        x.p_ref = x.p_new = true;
        x.p_exact = pinned;
    } else {
        x.s_ref = true;
        x.s_exact = pinned;
        if (pinned) x.s = f;
    }
}

// an undecided check, one block: narrow the interval of s (and of the
// previous delta when it straddles too), then form the serial sums where
// that still does not decide; every thread of the block (out of line: the
// iteration kernels' register allocation is not shaped by it)
template <int NT>
__device__ __noinline__ void serial_form(SerialCheck &x, const LoopyCtl *c, const float *absdiff, float *buf,
                                         uint32_t cap, bool narrow) {
    const uint64_t n = c->n_terms, stride = c->ad_stride;
    const uint32_t pb = c->prev_buf;
    const float tol = c->tol;
    double lo, hi;
    if (narrow) {
        ++x.refines;
        if (refine_block<NT>(absdiff + (size_t)x.cb * stride, n, buf, cap, lo, hi)) serial_narrow(x, 0, lo, hi);
        x.d = serial_decide(x.lo, x.hi, x.s_exact, x.plo, x.phi, x.p_exact, tol);
        if (x.d < 0 && !x.p_exact && !x.p_ref) {
            if (refine_block<NT>(absdiff + (size_t)pb * stride, n, buf, cap, lo, hi)) serial_narrow(x, 1, lo, hi);
            x.d = serial_decide(x.lo, x.hi, x.s_exact, x.plo, x.phi, x.p_exact, tol);
        }
    }
    if (x.d < 0 && !x.s_exact) {
        x.s = exact_serial_sum<NT>(absdiff + (size_t)x.cb * stride, n, buf, cap);
        x.lo = x.hi = (double)x.s;
        x.s_exact = true;
        ++x.sums;
        x.d = serial_decide(x.lo, x.hi, true, x.plo, x.phi, x.p_exact, tol);
    }
    if (x.d < 0) {
        const float p = exact_serial_sum<NT>(absdiff + (size_t)pb * stride, n, buf, cap);
        x.plo = x.phi = (double)p;
        x.p_exact = x.p_new = true;
        ++x.sums;
        x.d = serial_decide(x.lo, x.hi, true, x.plo, x.phi, true, tol);
    }
}

// record the check and run the loop bookkeeping; one thread
__device__ void serial_commit(LoopyCtl *c, const SerialCheck &x) {
    if (x.p_new) {
        c->plo = x.plo;
        c->phi = x.phi;
        c->prev_ref = x.p_ref ? 1u : 0u;
        if (x.p_exact) {
            c->prev_f = (float)x.plo;
            c->prev_exact = 1;
        }
    }
    c->dlo = x.lo;
    c->dhi = x.hi;
    c->delta_exact = x.s_exact ? 1u : 0u;
    c->delta_ref = x.s_ref ? 1u : 0u;
    c->cur_buf = x.cb;
    c->serial_sums += x.sums;
    c->serial_refines += x.refines;
    finalize_with(c, true, x.d == 1, x.s, x.T);
}

// T (valid in thread 0, as block_sum leaves it) to every thread
__device__ __forceinline__ double broadcast_sum(double T) {
    __shared__ double s_T;
    if (threadIdx.x == 0) s_T = T;
    __syncthreads();
    T = s_T;
    __syncthreads();
    return T;
}

// serial-mode decision and bookkeeping by one block after a check whose f64
// term sum is T; every thread of the block calls it and takes the same
// branches, thread 0 writes c
template <int NT>
__device__ __noinline__ void finalize_serial(LoopyCtl *c, bool want, double T, const float *absdiff, float *buf,
                                             uint32_t cap) {
    if (!want) {
        if (threadIdx.x == 0) finalize_with(c, false, false, 0.0f, 0.0);
        return;
    }
    SerialCheck x = serial_check(c, broadcast_sum(T));
    if (x.d < 0) serial_form<NT>(x, c, absdiff, buf, cap, true);
    __syncthreads();   // every thread has read c
    if (threadIdx.x == 0) serial_commit(c, x);
}

// grid-wide deterministic delta: per-block partial, last block sums the
// partials in a fixed order and finalizes.  In serial mode the last block
// decides from the f64 sum and, when the bound cannot, sums the terms every
// block wrote to absdiff (a fence per writer makes them visible before the
// ticket); buf/cap: the block's shared staging buffer for that sum (floats).
template <int NT, bool SER = false>
__device__ __forceinline__ void reduce_and_finalize(LoopyCtl *ctl, double *partials, double dsum, bool want,
                                                    double *red, bool *s_last, const float *absdiff = nullptr,
                                                    float *buf = nullptr, uint32_t cap = 0) {
    if (SER && want) __threadfence();
    double t = block_sum<NT>(dsum, red);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = t;
        // release: the partial is visible before the ticket is
        unsigned ticket;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(ticket) : "l"(&ctl->counter) : "memory");
        *s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (*s_last) {
        __threadfence();
        double acc = 0.0;
        for (uint32_t k = threadIdx.x; k < gridDim.x; k += NT) acc += __ldcg(partials + k);
        double tot = block_sum<NT>(acc, red);
        if constexpr (SER) {
            finalize_serial<NT>(ctl, want, tot, absdiff, buf, cap);
            if (threadIdx.x == 0) ctl->counter = 0;
        } else if (threadIdx.x == 0) {
            ctl->counter = 0;
            finalize(ctl, want, (float)tot, tot);
        }
    }
}

// this check's |diff| buffer (serial mode), else nullptr
__device__ __forceinline__ float *check_buffer(const LoopyCtl *c, float *absdiff, uint32_t it, bool want) {
    if (!c->serial || !want) return nullptr;
    return absdiff + (size_t)(check_index(it, c->check_every) % 3u) * c->ad_stride;
}

// one 256-node tile of the flooding iteration (see the file header)
template <int MS, bool UNI, int FU>
__device__ __forceinline__ void flood_tile(const FloodArgs &a, uint32_t tile, bool want, float *__restrict__ absd,
                                           const float *__restrict__ m_old, float *__restrict__ m_new,
                                           const float *__restrict__ q_in, float *__restrict__ q_out, uint64_t keep,
                                           float *sm, double &dsum) {
    constexpr int NT = flood_nt<MS>();
    constexpr uint32_t EMAX = flood_smem_floats<MS>() / MS;
    const uint32_t V = a.V, tid = threadIdx.x, v0 = a.v_base + tile * NT;
    const uint32_t vend = min(v0 + NT, V);
    const uint32_t e0 = a.in_ptr[v0], e1 = a.in_ptr[vend];
    const uint32_t v = v0 + tid;
    const bool has = v < V;
    uint32_t r0 = 0, r1 = 0;
    int S = MS;
    float b[MS];
    if (has) {
        r0 = a.in_ptr[v];
        r1 = a.in_ptr[v + 1];
        if (!UNI) S = a.node_s[v];
        ldv<MS, kStream>(a.belief + (size_t)v * MS, b);
    }
    float prod[MS];
#pragma unroll
    for (int i = 0; i < MS; ++i) prod[i] = 1.0f;

    for (uint32_t c0 = e0; c0 < e1; c0 += EMAX) {
        const uint32_t c1 = min(e1, c0 + EMAX);
        // phase 1: messages of this chunk of in-edges, FU edges per thread per
        // round with every load of the round issued before the first use, so
        // a thread keeps FU gathers in flight instead of one
        if (FU == 1 && a.pipe) {
            // software pipeline, one in-edge per thread per round: the next
            // round's source id (and with pipe 2 its table and old message)
            // is in flight while this round's gather completes
            uint32_t p = c0 + tid;
            uint32_t s_cur = p < c1 ? __ldcs(a.in_src + p) : 0u;
            float j_cur[MS * MS], o_cur[MS];
            const bool deep = a.pipe >= 2 && MS <= 2;
            if (deep && p < c1) {
                ldv<MS * MS, kStream>(a.joint + (size_t)p * (MS * MS), j_cur);
                if (want) ldv<MS, kStream>(m_old + (size_t)p * MS, o_cur);
            }
            for (; p < c1; p += NT) {
                const uint32_t pn = p + NT;
                const uint32_t s_nxt = pn < c1 ? __ldcs(a.in_src + pn) : 0u;
                int x = MS, y = MS;
                if (!UNI) {
                    const uint8_t d = a.pos_dims[p];
                    x = d & 15;
                    y = d >> 4;
                }
                float q[MS], m[MS], o[MS];
                if (s_cur < a.hot) ldv_pol<MS>(q_in + (size_t)s_cur * MS, q, keep);
                else ldv<MS>(q_in + (size_t)s_cur * MS, q);
                if (deep) {
#pragma unroll
                    for (int k = 0; k < MS; ++k) o[k] = o_cur[k];
                    float jt[MS * MS];
#pragma unroll
                    for (int k = 0; k < MS * MS; ++k) jt[k] = j_cur[k];
                    if (pn < c1) {
                        ldv<MS * MS, kStream>(a.joint + (size_t)pn * (MS * MS), j_cur);
                        if (want) ldv<MS, kStream>(m_old + (size_t)pn * MS, o_cur);
                    }
                    send_msg_regs<MS, UNI>(jt, q, x, y, m);
                } else {
                    if (want) ldv<MS, kStream>(m_old + (size_t)p * MS, o);
                    send_msg<MS, UNI>(a.joint + (size_t)p * (MS * MS), q, x, y, m);
                }
                if (want) {
                    float ad[MS];
#pragma unroll
                    for (int k = 0; k < MS; ++k) {
                        float d = 0.0f;
                        if (UNI || k < x) {
                            d = FSUB(o[k], m[k]);
                            if (d != d) d = 0.0f;
                            d = fabsf(d);
                        }
                        ad[k] = d;
                        dsum += (double)d;
                    }
                    if (absd) stv<MS>(absd + (size_t)__ldg(a.pos_edge + p) * MS, ad);
                }
                stv<MS, kStream>(m_new + (size_t)p * MS, m);
                stv<MS>(sm + (size_t)(p - c0) * MS, m);
                s_cur = s_nxt;
            }
        } else
        for (uint32_t pb = c0 + tid; pb < c1; pb += NT * FU) {
            uint32_t src[FU];
            int x[FU], y[FU];
            float jt[FU][FU > 1 ? MS * MS : 1], o[FU][MS], q[FU][MS];
#pragma unroll
            for (int u = 0; u < FU; ++u) {
                const uint32_t p = pb + u * NT;
                src[u] = 0;
                x[u] = MS;
                y[u] = MS;
                if (p < c1) {
                    src[u] = __ldcs(a.in_src + p);
                    if (!UNI) {
                        const uint8_t d = a.pos_dims[p];
                        x[u] = d & 15;
                        y[u] = d >> 4;
                    }
                    if constexpr (FU > 1) ldv<MS * MS, kStream>(a.joint + (size_t)p * (MS * MS), jt[u]);
                    if (want) ldv<MS, kStream>(m_old + (size_t)p * MS, o[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < FU; ++u)
                if (pb + u * NT < c1) {
                    if (src[u] < a.hot) ldv_pol<MS>(q_in + (size_t)src[u] * MS, q[u], keep);
                    else ldv<MS>(q_in + (size_t)src[u] * MS, q[u]);
                }
#pragma unroll
            for (int u = 0; u < FU; ++u) {
                const uint32_t p = pb + u * NT;
                if (p >= c1) break;
                float m[MS];
                if constexpr (FU > 1) send_msg_regs<MS, UNI>(jt[u], q[u], x[u], y[u], m);
                else send_msg<MS, UNI>(a.joint + (size_t)p * (MS * MS), q[u], x[u], y[u], m);
                if (want) {
                    float ad[MS];
#pragma unroll
                    for (int k = 0; k < MS; ++k) {
                        float d = 0.0f;
                        if (UNI || k < x[u]) {
                            d = FSUB(o[u][k], m[k]);
                            if (d != d) d = 0.0f;
                            d = fabsf(d);
                        }
                        ad[k] = d;
                        dsum += (double)d;
                    }
                    if (absd) stv<MS>(absd + (size_t)__ldg(a.pos_edge + p) * MS, ad);
                }
                stv<MS, kStream>(m_new + (size_t)p * MS, m);
                stv<MS>(sm + (size_t)(p - c0) * MS, m);
            }
        }
        __syncthreads();
        // phase 2a: this node's product over its in-edges inside the chunk
        if (has) {
            const uint32_t lo = max(r0, c0), hi = min(r1, c1);
            for (uint32_t p = lo; p < hi; ++p) {
                float mm[MS];
                ldv<MS>(sm + (size_t)(p - c0) * MS, mm);
                combine<MS, UNI>(prod, mm, S);
            }
        }
        // the next chunk overwrites the messages; after the last chunk the
        // caller's barrier at the end of the tile does
        if (c1 < e1) __syncthreads();
    }

    // phase 2b: marginalise (graph.c:1003-1023), then the next send buffer
    // (graph.c:850-882) from the same messages
    if (has) {
        if (r1 > r0) {
#pragma unroll
            for (int i = 0; i < MS; ++i)
                if (UNI || i < S) b[i] = FMUL(b[i], prod[i]);
        }
        normalise<MS, UNI>(b, S);
        stv<MS, kStream>(a.belief + (size_t)v * MS, b);
        float qo[MS];
#pragma unroll
        for (int i = 0; i < MS; ++i) qo[i] = b[i];
        if (e1 - e0 <= EMAX) {
            for (uint32_t p = r0; p < r1; ++p) {
                float mm[MS];
                ldv<MS>(sm + (size_t)(p - e0) * MS, mm);
                combine<MS, UNI>(qo, mm, S);
            }
        } else {
            for (uint32_t p = r0; p < r1; ++p) {
                float mm[MS];
                ldv<MS>(m_new + (size_t)p * MS, mm);
                combine<MS, UNI>(qo, mm, S);
            }
        }
        if (v < a.hot) stv_pol<MS>(q_out + (size_t)v * MS, qo, keep);
        else stv<MS>(q_out + (size_t)v * MS, qo);
    }

}

// Tiles are taken round-robin (tile = blockIdx.x + k * gridDim.x, a fixed
// assignment, so the delta sums in a fixed order); with ntiles == gridDim.x
// each block takes one tile.  A persistent grid (resident blocks per SM x SMs)
// pays the block's delta reduction and ticket once instead of per tile.
template <int MS, bool UNI, int FU, int MB = flood_min_blocks<MS, FU>(), bool SER = false>
__global__ void __launch_bounds__(flood_nt<MS>(), MB) k_flood(const FloodArgs a, uint32_t ntiles) {
    constexpr int NT = flood_nt<MS>();
    constexpr uint32_t EMAX = flood_smem_floats<MS>() / MS;
    __shared__ __align__(16) float sm[EMAX * MS];
    __shared__ double red[NT / 32];
    __shared__ bool s_last;

    LoopyCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint32_t it = ctl->it, ce = ctl->check_every;
    const bool want = (ce <= 1) || ((it + 1) % ce == 0);
    const int mp = (int)((ctl->msg_parity0 + it) & 1u), qp = (int)((ctl->q_parity0 + it) & 1u);
    const float *__restrict__ m_old = mp ? a.msg1 : a.msg0;
    float *__restrict__ m_new = mp ? a.msg0 : a.msg1;
    const float *__restrict__ q_in = qp ? a.q1 : a.q0;
    float *__restrict__ q_out = qp ? a.q0 : a.q1;
    const uint64_t keep = l2_evict_last_policy();
    // serial delta (SER): the |diff| terms go to this check's buffer
    float *absd = SER ? check_buffer(ctl, a.absdiff, it, want) : nullptr;
    double dsum = 0.0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        flood_tile<MS, UNI, FU>(a, tile, want, absd, m_old, m_new, q_in, q_out, keep, sm, dsum);
        __syncthreads();   // the tile's messages in shared memory are consumed
    }
    reduce_and_finalize<NT, SER>(ctl, a.partials, dsum, want, red, &s_last, a.absdiff, sm, EMAX * MS);
}

// Small graphs: every iteration in one cooperative launch.  When each tile
// has a block of its own on the GPU at once (a cooperative launch guarantees
// co-residency), the per-iteration launch costs more than the iteration, so
// the blocks loop over the iterations themselves and meet at a grid barrier
// after each one (its wait bounded by kWaitNs; a block that gives up sets
// bar_fail, and the others then give up at the next barrier).  Each block
// keeps a copy of the control block and, after the barrier, sums the
// per-block delta partials in the same fixed order as k_flood's last block
// does, so every block takes the same stopping decision and the results equal
// the one-launch-per-iteration loop's.  Partials are double-buffered by
// iteration parity: a block writes the next iteration's while others may
// still read this one's.
constexpr uint64_t kBarrierWaitNs = 2000000000ull;   // 2 s

// The wait is bounded by kBarrierWaitNs, or by c->wait_ms when the host set
// one.  Test hook: with c->bar_skip == blockIdx.x + 1 this block does not
// arrive at the first barrier (gen 0) and goes on, so the other blocks' waits
// run out and the run ends with bar_fail; every later wait of this block is
// bounded the same way, so the launch still ends.
__device__ __forceinline__ bool grid_barrier(LoopyCtl *c, uint32_t &gen, uint32_t *s_fail) {
    __syncthreads();
    if (threadIdx.x == 0 && !*s_fail && !(gen == 0 && c->bar_skip == blockIdx.x + 1u)) {
        const uint32_t g0 = gen;
        const uint64_t limit = c->wait_ms ? (uint64_t)c->wait_ms * 1000000ull : kBarrierWaitNs;
        __threadfence();
        if (atomicAdd(&c->bar_count, 1u) == gridDim.x - 1) {
            c->bar_count = 0;   // untouched until the generation moves
            __threadfence();
            atomicExch(&c->bar_gen, g0 + 1u);
        } else {
            const uint64_t t0 = global_ns();
            while (*(volatile uint32_t *)&c->bar_gen == g0) {
                if (global_ns() - t0 > limit) {
                    *s_fail = 1;
                    atomicExch(&c->bar_fail, 1u);
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
    gen += 1;
    return *s_fail == 0;
}

// the narrowed intervals of an undecided check in the one-launch loop,
// grid-wide: each block takes one slice of the terms (of s, and of the
// previous delta when that is neither exact nor narrowed yet); slice sums,
// a barrier, each slice's errors from its exact prefix, a barrier, and
// every block sums the same slices in the same order, so all blocks end with
// the same intervals.  Scratch: 8 doubles per block after the partials.
// false when a barrier gave up.
template <int NT>
__device__ bool grid_refine(const FloodArgs &a, LoopyCtl *ctl, uint32_t &gen, uint32_t *s_fail, SerialCheck &x,
                            const LoopyCtl &sc, float *buf, uint32_t cap, double *red) {
    __shared__ double s_b[4];
    __shared__ double s_v[NT / 32][6];
    __shared__ double s_t[6];
    const uint64_t n = sc.n_terms, stride = sc.ad_stride;
    const double c0 = refine_c0(n);
    if (c0 == 0.0) return true;
    const bool do_p = !x.p_exact && !x.p_ref;
    ++x.refines;
    const uint32_t G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    double *scr = a.partials + 2 * (size_t)G;
    const uint64_t L = ((n + G - 1) / G + 3) & ~3ull;
    const uint64_t lo = min(n, (uint64_t)b * L), hi = min(n, lo + L);
    const float *xs = a.absdiff + (size_t)x.cb * stride, *xp = a.absdiff + (size_t)sc.prev_buf * stride;
    double ls = 0.0, lp = 0.0;
    for (uint64_t k = lo + tid; k < hi; k += NT) {
        ls += (double)__ldcg(xs + k);
        if (do_p) lp += (double)__ldcg(xp + k);
    }
    ls = block_sum<NT>(ls, red);
    lp = block_sum<NT>(lp, red);
    if (tid == 0) {
        scr[b] = ls;
        scr[G + b] = lp;
    }
    if (!grid_barrier(ctl, gen, s_fail)) return false;
    // prefixes before this slice, and the totals (the same in every block)
    double ps = 0.0, ts = 0.0, pp = 0.0, tp = 0.0;
    for (uint32_t k = tid; k < G; k += NT) {
        const double vs = __ldcg(scr + k), vp = __ldcg(scr + G + k);
        ts += vs;
        tp += vp;
        if (k < b) {
            ps += vs;
            pp += vp;
        }
    }
    ps = block_sum<NT>(ps, red);
    ts = block_sum<NT>(ts, red);
    pp = block_sum<NT>(pp, red);
    tp = block_sum<NT>(tp, red);
    if (tid == 0) {
        s_b[0] = ps;
        s_b[1] = ts;
        s_b[2] = pp;
        s_b[3] = tp;
    }
    __syncthreads();
    ps = s_b[0];
    ts = s_b[1];
    pp = s_b[2];
    tp = s_b[3];
    double pe;
    const Refine rs = refine_segment<NT>(xs, lo, hi, ps, c0, buf, cap, pe);
    Refine rp{0.0, 0.0, 0.0, false};
    if (do_p) rp = refine_segment<NT>(xp, lo, hi, pp, c0, buf, cap, pe);
    const double inf = __longlong_as_double(0x7ff0000000000000ll);
    if (tid == 0) {
        scr[2 * (size_t)G + b] = rs.E;
        scr[3 * (size_t)G + b] = rs.A;
        scr[4 * (size_t)G + b] = rs.bad ? inf : rs.B;
        scr[5 * (size_t)G + b] = rp.E;
        scr[6 * (size_t)G + b] = rp.A;
        scr[7 * (size_t)G + b] = rp.bad ? inf : rp.B;
    }
    if (!grid_barrier(ctl, gen, s_fail)) return false;
    // the same totals in every block: fixed per-thread slices, then a fixed
    // reduction order; the bounds (j = 2, 5) rounded up
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    for (uint32_t k = tid; k < G; k += NT) {
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            const double y = __ldcg(scr + (size_t)(2 + j) * G + k);
            v[j] = (j == 2 || j == 5) ? __dadd_ru(v[j], y) : v[j] + y;
        }
    }
#pragma unroll
    for (int j = 0; j < 6; ++j)
        for (int d = 16; d > 0; d >>= 1) {
            const double y = __shfl_xor_sync(0xffffffffu, v[j], d);
            v[j] = (j == 2 || j == 5) ? __dadd_ru(v[j], y) : v[j] + y;
        }
    if ((tid & 31u) == 0u)
        for (int j = 0; j < 6; ++j) s_v[tid >> 5][j] = v[j];
    __syncthreads();
    if (tid == 0)
        for (int j = 0; j < 6; ++j) {
            double t = 0.0;
            for (int w = 0; w < NT / 32; ++w) t = (j == 2 || j == 5) ? __dadd_ru(t, s_v[w][j]) : t + s_v[w][j];
            s_t[j] = t;
        }
    __syncthreads();
    double lo2, hi2;
    const Refine Rs{s_t[0], s_t[1], s_t[2], !(s_t[2] < inf)};
    if (!Rs.bad) {
        refine_interval(ts, Rs, n, lo2, hi2);
        serial_narrow(x, 0, lo2, hi2);
    }
    if (do_p) {
        const Refine Rp{s_t[3], s_t[4], s_t[5], !(s_t[5] < inf)};
        if (!Rp.bad) {
            refine_interval(tp, Rp, n, lo2, hi2);
            serial_narrow(x, 1, lo2, hi2);
        }
    }
    x.d = serial_decide(x.lo, x.hi, x.s_exact, x.plo, x.phi, x.p_exact, sc.tol);
    __syncthreads();   // s_t and s_b are free
    return true;
}

template <int MS, bool UNI, int FU, bool SER = false, int MB = flood_min_blocks<MS, FU>()>
__global__ void __launch_bounds__(flood_nt<MS>(), MB) k_flood_fused(const FloodArgs a, uint32_t ntiles) {
    constexpr int NT = flood_nt<MS>();
    constexpr uint32_t EMAX = flood_smem_floats<MS>() / MS;
    __shared__ __align__(16) float sm[EMAX * MS];
    __shared__ double red[NT / 32];
    __shared__ LoopyCtl s_ctl;
    __shared__ uint32_t s_fail;

    LoopyCtl *ctl = a.ctl;
    if (threadIdx.x == 0) {
        s_ctl = *ctl;
        s_fail = 0;
    }
    __syncthreads();
    const uint64_t keep = l2_evict_last_policy();
    uint32_t gen = 0;
    while (!s_ctl.done) {
        const uint32_t it = s_ctl.it, ce = s_ctl.check_every;
        const bool want = (ce <= 1) || ((it + 1) % ce == 0);
        const int mp = (int)((s_ctl.msg_parity0 + it) & 1u), qp = (int)((s_ctl.q_parity0 + it) & 1u);
        const float *__restrict__ m_old = mp ? a.msg1 : a.msg0;
        float *__restrict__ m_new = mp ? a.msg0 : a.msg1;
        const float *__restrict__ q_in = qp ? a.q1 : a.q0;
        float *__restrict__ q_out = qp ? a.q0 : a.q1;
        float *absd = SER ? check_buffer(&s_ctl, a.absdiff, it, want) : nullptr;
        double dsum = 0.0;
        for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            flood_tile<MS, UNI, FU>(a, tile, want, absd, m_old, m_new, q_in, q_out, keep, sm, dsum);
            __syncthreads();
        }
        const double t = block_sum<NT>(dsum, red);
        double *part = a.partials + (size_t)(it & 1u) * gridDim.x;
        if (threadIdx.x == 0) part[blockIdx.x] = t;
        if (!grid_barrier(ctl, gen, &s_fail)) break;
        double acc = 0.0;
        for (uint32_t k = threadIdx.x; k < gridDim.x; k += NT) acc += __ldcg(part + k);
        const double tot = block_sum<NT>(acc, red);
        if (SER && want) {
            // every block reaches the same decision from the same sum; when
            // the bound cannot decide, block 0 forms the serial sums and the
            // blocks meet once more to read them.  The terms are
            // triple-buffered by check, so no block overwrites them while
            // block 0 reads.
            SerialCheck x = serial_check(&s_ctl, broadcast_sum(tot));
            if (x.d < 0 && !grid_refine<NT>(a, ctl, gen, &s_fail, x, s_ctl, sm, EMAX * MS, red)) break;
            if (x.d < 0) {
                const bool s_ex0 = x.s_exact, p_ex0 = x.p_exact;
                if (blockIdx.x == 0) {
                    serial_form<NT>(x, &s_ctl, a.absdiff, sm, EMAX * MS, false);
                    if (threadIdx.x == 0) {
                        ctl->fb_s = x.s;
                        ctl->fb_p = (float)x.plo;
                        ctl->fb_pform = x.p_exact && !p_ex0;
                    }
                }
                if (!grid_barrier(ctl, gen, &s_fail)) break;
                if (blockIdx.x != 0) {
                    if (!s_ex0) {
                        x.s = *(volatile float *)&ctl->fb_s;
                        x.lo = x.hi = (double)x.s;
                        x.s_exact = true;
                    }
                    if (*(volatile uint32_t *)&ctl->fb_pform) {
                        x.plo = x.phi = (double)*(volatile float *)&ctl->fb_p;
                        x.p_exact = x.p_new = true;
                    }
                    x.d = serial_decide(x.lo, x.hi, x.s_exact, x.plo, x.phi, x.p_exact, s_ctl.tol);
                }
            }
            __syncthreads();
            if (threadIdx.x == 0) serial_commit(&s_ctl, x);
        } else if (threadIdx.x == 0) {
            finalize(&s_ctl, want, (float)tot, tot);
        }
        __syncthreads();
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && !s_fail) {
        ctl->it = s_ctl.it;
        ctl->ret = s_ctl.ret;
        ctl->num_iter = s_ctl.num_iter;
        ctl->final_i = s_ctl.final_i;
        ctl->delta_f = s_ctl.delta_f;
        ctl->prev_f = s_ctl.prev_f;
        ctl->delta_d = s_ctl.delta_d;
        ctl->prev_d = s_ctl.prev_d;
        ctl->dlo = s_ctl.dlo;
        ctl->dhi = s_ctl.dhi;
        ctl->plo = s_ctl.plo;
        ctl->phi = s_ctl.phi;
        ctl->delta_exact = s_ctl.delta_exact;
        ctl->prev_exact = s_ctl.prev_exact;
        ctl->cur_buf = s_ctl.cur_buf;
        ctl->prev_buf = s_ctl.prev_buf;
        ctl->serial_sums = s_ctl.serial_sums;
        ctl->serial_refines = s_ctl.serial_refines;
        ctl->delta_ref = s_ctl.delta_ref;
        ctl->prev_ref = s_ctl.prev_ref;
        __threadfence();
        ctl->done = s_ctl.done;
    }
}

// Staged form of k_flood for uniform 2-state graphs (the layout is written
// for 2 or 4 states; 4-state tables do not leave room for two stages of a
// 256-node tile).  A persistent
// grid walks the 256-node tiles round-robin (tile = blockIdx.x + k*gridDim.x,
// a fixed assignment, so the delta sums in a fixed order).  For each tile one
// thread issues bulk asynchronous copies (cp.async.bulk, no multicast) of the
// tile's contiguous streams -- row pointers, beliefs, source ids, tables and
// the previous messages -- into a ring of shared-memory stages, ST tiles
// ahead of the tile being computed, each stage completing on its mbarrier.
// The threads then only gather Q[src] (the one random access) and do the
// arithmetic, in the order and rounding of k_flood.  A tile whose in-edges
// do not fit a stage (more than CAP) is computed from global memory in
// CAP-edge chunks, as k_flood does.
//
// Bulk copies need 16-byte aligned ranges: each stream is copied from its
// first element rounded down to a 16-byte boundary and for a length rounded
// up, so the graph's arrays carry padding past their ends (engine.cu,
// kArrayPadNodes / kArrayPadEdges).
constexpr uint32_t kStagedTN = 256;      // nodes per tile = threads per CTA
constexpr uint64_t kWaitNs = 2000000000ull;  // bound on one stage wait: 2 s

__host__ __device__ constexpr uint32_t round16(uint32_t b) { return (b + 15u) & ~15u; }

template <int MS>
struct Staged {
    static constexpr uint32_t TN = kStagedTN;
    static constexpr uint32_t CAP = MS <= 2 ? 1536 : 768;   // in-edges per stage
    static constexpr int ST = 2;                            // stages
    static constexpr int FU = MS <= 2 ? 4 : 2;              // gathers in flight per thread
    static constexpr uint32_t EPM = 16 / (MS * 4);          // edges per 16 B of messages
    // stage layout (byte offsets, each a multiple of 16)
    static constexpr uint32_t SRC = 0;                                  // CAP + 8 u32
    static constexpr uint32_t JNT = SRC + (CAP + 8) * 4;                // CAP tables
    static constexpr uint32_t MOLD = JNT + CAP * MS * MS * 4;           // CAP + 2*EPM messages
    static constexpr uint32_t PTR = MOLD + round16((CAP + 2 * EPM) * MS * 4);  // TN + 4 u32
    static constexpr uint32_t BEL = PTR + (TN + 4) * 4;                 // TN beliefs
    static constexpr uint32_t STAGE = round16(BEL + TN * MS * 4);
    // after the stages: the tile's new messages, then the mbarriers
    static constexpr uint32_t MSG = ST * STAGE;
    static constexpr uint32_t BAR = MSG + round16(CAP * MS * 4);
    static constexpr uint32_t SMEM = BAR + 16 * ST;
    static_assert(MS == 2 || MS == 4, "staged tiles: 2 or 4 states");
    static_assert(CAP % 4 == 0 && TN % 4 == 0, "16-byte aligned stage sections");
};

// issue the copies of `tile` into stage `st` (one thread); the byte count the
// mbarrier expects is the sum of exactly the copies issued
template <int MS>
__device__ void staged_issue(const FloodArgs &a, const float *m_old, bool want, uint32_t tile, unsigned char *st,
                             uint64_t *bar) {
    using C = Staged<MS>;
    const uint32_t v0 = tile * C::TN, v1 = min(v0 + C::TN, a.V);
    const uint32_t e0 = a.in_ptr[v0], e1 = a.in_ptr[v1];
    const uint32_t b_ptr = (C::TN + 4) * 4, b_bel = C::TN * MS * 4;
    uint32_t b_src = 0, b_j = 0, b_m = 0, a4 = 0, am = 0;
    if (e1 > e0 && e1 - e0 <= C::CAP) {
        a4 = e0 & ~3u;
        b_src = ((e1 - a4 + 3u) & ~3u) * 4;
        b_j = (e1 - e0) * MS * MS * 4;
        if (want) {
            am = e0 & ~(C::EPM - 1);
            b_m = ((e1 - am + C::EPM - 1) & ~(C::EPM - 1)) * MS * 4;
        }
    }
    mbar_arrive_expect_tx(bar, b_ptr + b_bel + b_src + b_j + b_m);
    bulk_g2s(st + C::PTR, a.in_ptr + v0, b_ptr, bar);
    bulk_g2s(st + C::BEL, a.belief + (size_t)v0 * MS, b_bel, bar);
    if (b_src) bulk_g2s(st + C::SRC, a.in_src + a4, b_src, bar);
    if (b_j) bulk_g2s(st + C::JNT, a.joint + (size_t)e0 * (MS * MS), b_j, bar);
    if (b_m) bulk_g2s(st + C::MOLD, m_old + (size_t)am * MS, b_m, bar);
}

template <int MS>
__global__ void __launch_bounds__(kStagedTN) k_flood_staged(const FloodArgs a, uint32_t ntiles) {
    using C = Staged<MS>;
    constexpr uint32_t NT = C::TN;
    constexpr int FU = C::FU;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ double red[NT / 32];
    __shared__ bool s_last;
    __shared__ uint32_t s_err;

    LoopyCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint32_t it = ctl->it, ce = ctl->check_every;
    const bool want = (ce <= 1) || ((it + 1) % ce == 0);
    const int mp = (int)((ctl->msg_parity0 + it) & 1u), qp = (int)((ctl->q_parity0 + it) & 1u);
    const float *__restrict__ m_old = mp ? a.msg1 : a.msg0;
    float *__restrict__ m_new = mp ? a.msg0 : a.msg1;
    const float *__restrict__ q_in = qp ? a.q1 : a.q0;
    float *__restrict__ q_out = qp ? a.q0 : a.q1;
    const uint64_t keep = l2_evict_last_policy();
    const uint32_t tid = threadIdx.x;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + C::BAR);
    float *msg_s = reinterpret_cast<float *>(smem + C::MSG);

    if (tid == 0) {
        s_err = 0;
        for (int i = 0; i < C::ST; ++i) mbar_init(bars + i, 1);
        fence_mbar_init();
        for (int i = 0; i < C::ST; ++i) {
            const uint32_t t = blockIdx.x + (uint32_t)i * gridDim.x;
            if (t < ntiles) staged_issue<MS>(a, m_old, want, t, smem + i * C::STAGE, bars + i);
        }
    }
    __syncthreads();

    double dsum = 0.0;
    uint32_t k = 0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++k) {
        const int si = (int)(k % C::ST);
        const uint32_t par = (k / C::ST) & 1u;
        unsigned char *st = smem + si * C::STAGE;
        if (tid == 0 && !mbar_wait_bounded(bars + si, par, kWaitNs)) s_err = 1;
        __syncthreads();
        if (s_err) break;
        mbar_try_wait(bars + si, par);   // completed: orders this thread's reads after the copies

        const uint32_t *ptr_s = reinterpret_cast<const uint32_t *>(st + C::PTR);
        const uint32_t v0 = tile * NT, n = min(NT, a.V - v0);
        const uint32_t e0 = ptr_s[0], e1 = ptr_s[n];
        const bool staged = e1 - e0 <= C::CAP;
        const uint32_t v = v0 + tid;
        const bool has = tid < n;
        uint32_t r0 = 0, r1 = 0;
        if (has) {
            r0 = ptr_s[tid];
            r1 = ptr_s[tid + 1];
        }
        float prod[MS];
#pragma unroll
        for (int i = 0; i < MS; ++i) prod[i] = 1.0f;

        for (uint32_t c0 = e0; c0 < e1; c0 += C::CAP) {
            const uint32_t c1 = min(e1, c0 + C::CAP);
            if (staged) {
                const uint32_t *src_s = reinterpret_cast<const uint32_t *>(st + C::SRC) - (e0 & ~3u);
                const float *j_s = reinterpret_cast<const float *>(st + C::JNT) - (size_t)e0 * (MS * MS);
                const float *mo_s = reinterpret_cast<const float *>(st + C::MOLD) - (size_t)(e0 & ~(C::EPM - 1)) * MS;
                for (uint32_t pb = c0 + tid; pb < c1; pb += NT * FU) {
                    float q[FU][MS];
#pragma unroll
                    for (int u = 0; u < FU; ++u) {
                        const uint32_t p = pb + u * NT;
                        if (p < c1) {
                            const uint32_t sv = src_s[p];
                            if (sv < a.hot) ldv_pol<MS>(q_in + (size_t)sv * MS, q[u], keep);
                            else ldv<MS>(q_in + (size_t)sv * MS, q[u]);
                        }
                    }
#pragma unroll
                    for (int u = 0; u < FU; ++u) {
                        const uint32_t p = pb + u * NT;
                        if (p >= c1) break;
                        float jt[MS * MS], m[MS];
                        ldv<MS * MS>(j_s + (size_t)p * (MS * MS), jt);
                        send_msg_regs<MS, true>(jt, q[u], MS, MS, m);
                        if (want) {
                            float o[MS];
                            ldv<MS>(mo_s + (size_t)p * MS, o);
#pragma unroll
                            for (int kk = 0; kk < MS; ++kk) {
                                float d = FSUB(o[kk], m[kk]);
                                if (d != d) d = 0.0f;
                                dsum += (double)fabsf(d);
                            }
                        }
                        stv<MS, kStream>(m_new + (size_t)p * MS, m);
                        stv<MS>(msg_s + (size_t)(p - c0) * MS, m);
                    }
                }
            } else {
                for (uint32_t p = c0 + tid; p < c1; p += NT) {
                    const uint32_t sv = __ldcs(a.in_src + p);
                    float q[MS], m[MS];
                    if (sv < a.hot) ldv_pol<MS>(q_in + (size_t)sv * MS, q, keep);
                    else ldv<MS>(q_in + (size_t)sv * MS, q);
                    send_msg<MS, true>(a.joint + (size_t)p * (MS * MS), q, MS, MS, m);
                    if (want) {
                        float o[MS];
                        ldv<MS, kStream>(m_old + (size_t)p * MS, o);
#pragma unroll
                        for (int kk = 0; kk < MS; ++kk) {
                            float d = FSUB(o[kk], m[kk]);
                            if (d != d) d = 0.0f;
                            dsum += (double)fabsf(d);
                        }
                    }
                    stv<MS, kStream>(m_new + (size_t)p * MS, m);
                    stv<MS>(msg_s + (size_t)(p - c0) * MS, m);
                }
            }
            __syncthreads();
            if (has) {
                const uint32_t lo = max(r0, c0), hi = min(r1, c1);
                for (uint32_t p = lo; p < hi; ++p) {
                    float mm[MS];
                    ldv<MS>(msg_s + (size_t)(p - c0) * MS, mm);
                    combine<MS, true>(prod, mm, MS);
                }
            }
            __syncthreads();
        }

        if (has) {
            float b[MS];
            ldv<MS>(reinterpret_cast<const float *>(st + C::BEL) + (size_t)tid * MS, b);
            if (r1 > r0) {
#pragma unroll
                for (int i = 0; i < MS; ++i) b[i] = FMUL(b[i], prod[i]);
            }
            normalise<MS, true>(b, MS);
            stv<MS, kStream>(a.belief + (size_t)v * MS, b);
            float qo[MS];
#pragma unroll
            for (int i = 0; i < MS; ++i) qo[i] = b[i];
            if (staged) {
                for (uint32_t p = r0; p < r1; ++p) {
                    float mm[MS];
                    ldv<MS>(msg_s + (size_t)(p - e0) * MS, mm);
                    combine<MS, true>(qo, mm, MS);
                }
            } else {
                for (uint32_t p = r0; p < r1; ++p) {
                    float mm[MS];
                    ldv<MS>(m_new + (size_t)p * MS, mm);
                    combine<MS, true>(qo, mm, MS);
                }
            }
            if (v < a.hot) stv_pol<MS>(q_out + (size_t)v * MS, qo, keep);
            else stv<MS>(q_out + (size_t)v * MS, qo);
        }
        // every thread is done with the stage and the message buffer; the
        // stage takes the tile ST ahead
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0) {
            const uint32_t nt = tile + (uint32_t)C::ST * gridDim.x;
            if (nt < ntiles) staged_issue<MS>(a, m_old, want, nt, st, bars + si);
        }
    }

    if (s_err) {
        // a stage never completed: report it, wait (bounded) for the copies
        // still in flight into this CTA's stages, and leave the grid
        if (tid == 0) {
            atomicExch(&ctl->done, 3u);
            for (uint32_t j = 0; j < (uint32_t)C::ST; ++j) {
                const uint32_t kk = k + j, t = blockIdx.x + kk * gridDim.x;
                if (t < ntiles) mbar_wait_bounded(bars + (kk % C::ST), (kk / C::ST) & 1u, kWaitNs);
            }
        }
        return;
    }
    reduce_and_finalize<NT>(ctl, a.partials, dsum, want, red, &s_last);
}

#include "flood_split.cuh"

// Warp-tiled form of k_flood: each warp owns 32 consecutive destination
// nodes and their in-edges, so the two phases synchronise a warp instead of
// the block (the block meets once, for the delta).  Phase 1 issues the loads
// of U edges per lane before using any of them (source ids, tables and old
// messages first, then the dependent Q[src] gathers), so each warp keeps
// U times more bytes in flight; the node's belief is loaded at entry.  The
// arithmetic per value is k_flood's, in the same order.
template <int MS> constexpr uint32_t wflood_we() { return MS <= 2 ? 256 : (MS <= 4 ? 192 : 96); }
template <int MS> constexpr int wflood_unroll() { return MS <= 2 ? 4 : (MS <= 4 ? 2 : 1); }

template <int MS, bool UNI, int U>
__global__ void __launch_bounds__(256) k_flood_w(const FloodArgs a) {
    constexpr int NW = 8, NT = 256;
    constexpr uint32_t WE = wflood_we<MS>();
    constexpr bool JREG = MS * MS <= 16;
    __shared__ __align__(16) float sm[NW * WE * MS];
    __shared__ double red[NW];
    __shared__ bool s_last;

    LoopyCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint32_t it = ctl->it, ce = ctl->check_every;
    const bool serial = ctl->serial != 0;
    const bool want = (ce <= 1) || ((it + 1) % ce == 0);
    float *absd = check_buffer(ctl, a.absdiff, it, want);
    const int mp = (int)((ctl->msg_parity0 + it) & 1u), qp = (int)((ctl->q_parity0 + it) & 1u);
    const float *__restrict__ m_old = mp ? a.msg1 : a.msg0;
    float *__restrict__ m_new = mp ? a.msg0 : a.msg1;
    const float *__restrict__ q_in = qp ? a.q1 : a.q0;
    float *__restrict__ q_out = qp ? a.q0 : a.q1;

    const uint32_t V = a.V, lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    float *wsm = sm + warp * (WE * MS);
    const uint32_t v0 = (blockIdx.x * NW + warp) * 32u;
    double dsum = 0.0;
    if (v0 < V) {
        const uint32_t v = v0 + lane;
        const bool has = v < V;
        const uint32_t last = min(v0 + 32u, V) - 1u - v0;
        uint32_t r0 = 0, r1 = 0;
        int S = MS;
        float b[MS];
#pragma unroll
        for (int i = 0; i < MS; ++i) b[i] = 0.0f;
        if (has) {
            r0 = a.in_ptr[v];
            r1 = a.in_ptr[v + 1];
            if (!UNI) S = a.node_s[v];
            ldv<MS, kStream>(a.belief + (size_t)v * MS, b);
        }
        const uint32_t e0 = __shfl_sync(0xffffffffu, r0, 0);
        const uint32_t e1 = __shfl_sync(0xffffffffu, r1, last);
        float prod[MS];
#pragma unroll
        for (int i = 0; i < MS; ++i) prod[i] = 1.0f;

        for (uint32_t c0 = e0; c0 < e1; c0 += WE) {
            const uint32_t c1 = min(e1, c0 + WE);
            for (uint32_t base = c0 + lane; base < c1; base += 32u * U) {
                uint32_t src[U];
                float jr[JREG ? U : 1][JREG ? MS * MS : 1];
                float o[U][MS];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t p = base + 32u * u;
                    src[u] = 0;
                    if (p < c1) {
                        src[u] = __ldcs(a.in_src + p);
                        if constexpr (JREG) ldv<MS * MS, kStream>(a.joint + (size_t)p * (MS * MS), jr[u]);
                        if (want) ldv<MS, kStream>(m_old + (size_t)p * MS, o[u]);
                    }
                }
                float q[U][MS];
#pragma unroll
                for (int u = 0; u < U; ++u)
                    if (base + 32u * u < c1) ldv<MS>(q_in + (size_t)src[u] * MS, q[u]);
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const uint32_t p = base + 32u * u;
                    if (p >= c1) continue;
                    int x = MS, y = MS;
                    if (!UNI) {
                        const uint8_t d = a.pos_dims[p];
                        x = d & 15;
                        y = d >> 4;
                    }
                    float m[MS];
                    if constexpr (JREG) send_msg_regs<MS, UNI>(jr[u], q[u], x, y, m);
                    else send_msg<MS, UNI>(a.joint + (size_t)p * (MS * MS), q[u], x, y, m);
                    if (want) {
                        float ad[MS];
#pragma unroll
                        for (int k = 0; k < MS; ++k) {
                            float d = 0.0f;
                            if (UNI || k < x) {
                                d = FSUB(o[u][k], m[k]);
                                if (d != d) d = 0.0f;
                                d = fabsf(d);
                            }
                            ad[k] = d;
                            dsum += (double)d;
                        }
                        if (absd) stv<MS>(absd + (size_t)__ldg(a.pos_edge + p) * MS, ad);
                    }
                    stv<MS, kStream>(m_new + (size_t)p * MS, m);
                    stv<MS>(wsm + (size_t)(p - c0) * MS, m);
                }
            }
            __syncwarp();
            if (has) {
                const uint32_t lo = max(r0, c0), hi = min(r1, c1);
                for (uint32_t p = lo; p < hi; ++p) {
                    float mm[MS];
                    ldv<MS>(wsm + (size_t)(p - c0) * MS, mm);
                    combine<MS, UNI>(prod, mm, S);
                }
            }
            __syncwarp();
        }
        if (has) {
            if (r1 > r0) {
#pragma unroll
                for (int i = 0; i < MS; ++i)
                    if (UNI || i < S) b[i] = FMUL(b[i], prod[i]);
            }
            normalise<MS, UNI>(b, S);
            stv<MS, kStream>(a.belief + (size_t)v * MS, b);
            float qo[MS];
#pragma unroll
            for (int i = 0; i < MS; ++i) qo[i] = b[i];
            if (e1 - e0 <= WE) {
                for (uint32_t p = r0; p < r1; ++p) {
                    float mm[MS];
                    ldv<MS>(wsm + (size_t)(p - e0) * MS, mm);
                    combine<MS, UNI>(qo, mm, S);
                }
            } else {
                for (uint32_t p = r0; p < r1; ++p) {
                    float mm[MS];
                    ldv<MS>(m_new + (size_t)p * MS, mm);
                    combine<MS, UNI>(qo, mm, S);
                }
            }
            stv<MS>(q_out + (size_t)v * MS, qo);
        }
    }
    if (serial) reduce_and_finalize<NT, true>(ctl, a.partials, dsum, want, red, &s_last, a.absdiff, sm, NW * WE * MS);
    else reduce_and_finalize<NT>(ctl, a.partials, dsum, want, red, &s_last);
}

// One iteration for the destination nodes [a.v_base, a.V) only: a rank of a
// sharded run (one process per GPU, each owning a node range) computes its
// nodes' incoming messages from the full send buffers q_in, their beliefs
// and their next send buffers in q_out; the ranks then exchange q_out.  The
// per-tile work is k_flood's (flood_tile); the |diff| terms of the range are
// summed per block into `partials` and, by k_sum_partials, in a fixed order.
template <int MS, bool UNI, int FU>
__global__ void __launch_bounds__(flood_nt<MS>()) k_flood_range(const FloodArgs a, uint32_t ntiles,
                                                                const float *__restrict__ m_old,
                                                                float *__restrict__ m_new,
                                                                const float *__restrict__ q_in,
                                                                float *__restrict__ q_out, double *partials) {
    constexpr int NT = flood_nt<MS>();
    constexpr uint32_t EMAX = flood_smem_floats<MS>() / MS;
    __shared__ __align__(16) float sm[EMAX * MS];
    __shared__ double red[NT / 32];
    double dsum = 0.0;
    for (uint32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        flood_tile<MS, UNI, FU>(a, tile, true, nullptr, m_old, m_new, q_in, q_out, 0, sm, dsum);
        __syncthreads();
    }
    const double t = block_sum<NT>(dsum, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = t;
}

__global__ void k_sum_partials(const double *__restrict__ partials, uint32_t n, double *__restrict__ out) {
    __shared__ double red[8];
    double acc = 0.0;
    for (uint32_t k = threadIdx.x; k < n; k += 256) acc += partials[k];
    const double t = block_sum<256>(acc, red);
    if (threadIdx.x == 0) *out = t;
}

// prologue: Q_1 = b * prod of the latest messages (read_incoming_messages,
// graph.c:860-882, on the messages init_previous_edge left)
template <int MS, bool UNI>
__global__ void k_gather_q(uint32_t V, const uint32_t *__restrict__ in_ptr, const uint8_t *__restrict__ node_s,
                           const float *__restrict__ belief, const float *__restrict__ msg, float *__restrict__ q) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const int S = UNI ? MS : node_s[v];
    float b[MS];
    ldv<MS>(belief + (size_t)v * MS, b);
    for (uint32_t p = in_ptr[v]; p < in_ptr[v + 1]; ++p) {
        float mm[MS];
        ldv<MS>(msg + (size_t)p * MS, mm);
        combine<MS, UNI>(b, mm, S);
    }
    stv<MS>(q + (size_t)v * MS, b);
}

// init_previous_edge (graph.c:725-751): every edge carries normalise(J . b_src)
template <int MS, bool UNI>
__global__ void k_send_from_beliefs(uint32_t E, const uint32_t *__restrict__ in_src,
                                    const uint8_t *__restrict__ pos_dims, const float *__restrict__ joint,
                                    const float *__restrict__ belief, float *__restrict__ msg) {
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= E) return;
    const uint32_t s = in_src[p];
    int x = MS, y = MS;
    if (!UNI) {
        const uint8_t d = pos_dims[p];
        x = d & 15;
        y = d >> 4;
    }
    float buf[MS], m[MS];
    ldv<MS>(belief + (size_t)s * MS, buf);
    send_msg<MS, UNI>(joint + p * (MS * MS), buf, x, y, m);
    stv<MS>(msg + p * MS, m);
}

// one block forms the serial fp32 sum of x[0, n): the parallel form with NT
// threads and cap floats of staging, or the one-thread chain
__global__ void __launch_bounds__(256) k_serial_sum_bounds(const float *__restrict__ x, uint64_t n, double *lohi) {
    __shared__ __align__(16) float buf[8192];
    double lo = 0.0, hi = __longlong_as_double(0x7ff0000000000000ll);
    refine_block<256>(x, n, buf, 8192, lo, hi);
    if (threadIdx.x == 0) {
        lohi[0] = lo;
        lohi[1] = hi;
    }
}

template <int NT>
__global__ void __launch_bounds__(NT) k_serial_sum(const float *__restrict__ x, uint64_t n, float *out, int chain,
                                                  uint32_t cap) {
    __shared__ __align__(16) float buf[8192];
    const float s = chain ? block_serial_sum_chain<NT>(x, n, buf, 4096) : block_serial_sum<NT>(x, n, buf, cap);
    if (threadIdx.x == 0) *out = s;
}

// the reference's `delta` and `previous_delta` at return (graph.c:1300-1318)
// where the loop decided from bounds without forming them: block 0 sums the
// last check's terms, block 1 the check's before (serial fp32, edge-id order)
__global__ void __launch_bounds__(1024) k_delta_final(LoopyCtl *ctl, const float *__restrict__ absdiff) {
    __shared__ __align__(16) float buf[2 * 4096];
    const LoopyCtl c = *ctl;
    if (!c.serial || c.done == 0 || c.done == 3 || c.bar_fail) return;
    const bool prev = blockIdx.x == 1;
    if (prev ? c.prev_exact : c.delta_exact) return;
    const uint32_t b = prev ? c.prev_buf : c.cur_buf;
    const float s = exact_serial_sum<1024>(absdiff + (size_t)b * c.ad_stride, c.n_terms, buf, 2 * 4096);
    if (threadIdx.x == 0) {
        if (prev) ctl->prev_f = s;
        else ctl->delta_f = s;
    }
}

// ------------------------------------------------------------------------
// Edge-centric schedule (loopy_propagate_until_edge, graph.c:1186-1276, and
// its _acc form, graph.c:1444-1547), reproduced with its quirks:
//  * copy: num_edges * MAX_STATES BYTES of current into previous
//    (graph.c:1211), i.e. the first 2.5E floats of the reference's padded
//    array; the _acc form copies every float;
//  * send from the beliefs themselves (no incoming product);
//  * combine: belief(dest) *= message for each edge in edge order, no NaN
//    check; the _acc form multiplies by the message of edge i, the batch's
//    first iteration index (graph.c:1485);
//  * normalise: node 0's belief, once per node with that node's state count
//    (the base pointer is passed, graph.c:1225, :1505).
struct EdgeArgs {
    uint32_t V, E;
    const uint32_t *in_ptr, *in_src, *pos_edge, *edge_pos;
    const uint8_t *node_s, *pos_dims;
    const float *joint;
    float *belief;
    float *msg0, *msg1;
    double *partials;
    float *absdiff;
    LoopyCtl *ctl;
    const uint32_t *run_len;
    const uint8_t *run_s;
    uint32_t nruns;
};

// previous/current roles: the _acc form swaps local pointers every iteration
__device__ __forceinline__ void edge_roles(const EdgeArgs &a, uint32_t it, float *&prev, float *&curr) {
    const LoopyCtl *c = a.ctl;
    int p = (int)(c->msg_parity0 & 1u);
    if (c->acc_edge && (it & 1u)) p ^= 1;
    prev = p ? a.msg1 : a.msg0;
    curr = p ? a.msg0 : a.msg1;
}

template <int MS>
__global__ void k_edge_copy(const EdgeArgs a) {
    if (*(volatile uint32_t *)&a.ctl->done) return;
    float *prev, *curr;
    edge_roles(a, a.ctl->it, prev, curr);
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t p = t / MS;
    if (p >= a.E) return;
    const uint32_t k = (uint32_t)(t % MS);
    if (a.ctl->acc_edge) {
        prev[t] = curr[t];
        return;
    }
    const uint64_t f = (uint64_t)a.pos_edge[p] * 10u + k;   // float index in the padded layout
    const uint64_t nbytes = (uint64_t)a.E * 10u;
    const uint64_t nfull = nbytes / 4u;
    if (f < nfull) {
        prev[t] = curr[t];
    } else if (f == nfull && (nbytes & 3u)) {
        const uint32_t keep = 0xffffffffu << (8u * (uint32_t)(nbytes & 3u));
        const uint32_t cb = __float_as_uint(curr[t]), pb = __float_as_uint(prev[t]);
        prev[t] = __uint_as_float((pb & keep) | (cb & ~keep));
    }
}

template <int MS, bool UNI>
__global__ void k_edge_send(const EdgeArgs a) {
    if (*(volatile uint32_t *)&a.ctl->done) return;
    float *prev, *curr;
    edge_roles(a, a.ctl->it, prev, curr);
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= a.E) return;
    const uint32_t s = a.in_src[p];
    int x = MS, y = MS;
    if (!UNI) {
        const uint8_t d = a.pos_dims[p];
        x = d & 15;
        y = d >> 4;
    }
    float buf[MS], m[MS];
    ldv<MS>(a.belief + (size_t)s * MS, buf);
    send_msg<MS, UNI>(a.joint + p * (MS * MS), buf, x, y, m);
    stv<MS>(curr + p * MS, m);
}

template <int MS, bool UNI>
__global__ void k_edge_combine(const EdgeArgs a) {
    if (*(volatile uint32_t *)&a.ctl->done) return;
    const uint32_t it = a.ctl->it;
    float *prev, *curr;
    edge_roles(a, it, prev, curr);
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= a.V) return;
    const int S = UNI ? MS : a.node_s[v];
    const uint32_t r0 = a.in_ptr[v], r1 = a.in_ptr[v + 1];
    if (r0 == r1) return;
    float b[MS];
    ldv<MS>(a.belief + (size_t)v * MS, b);
    if (a.ctl->acc_edge) {
        const uint32_t i_batch = (it / 10u) * 10u;
        if (i_batch >= a.E) return;
        float mm[MS];
        ldv<MS>(curr + (size_t)a.edge_pos[i_batch] * MS, mm);
        for (uint32_t p = r0; p < r1; ++p) {
#pragma unroll
            for (int i = 0; i < MS; ++i)
                if (UNI || i < S) b[i] = FMUL(b[i], mm[i]);
        }
    } else {
        for (uint32_t p = r0; p < r1; ++p) {
            float mm[MS];
            ldv<MS>(curr + (size_t)p * MS, mm);
#pragma unroll
            for (int i = 0; i < MS; ++i)
                if (UNI || i < S) b[i] = FMUL(b[i], mm[i]);
        }
    }
    stv<MS>(a.belief + (size_t)v * MS, b);
}

// node 0 normalised once per node, in node order; within a run of equal
// state counts the map is applied until it stops changing node 0 (it is then
// the identity for the rest of the run)
template <int MS>
__global__ void k_edge_normalise_node0(const EdgeArgs a) {
    if (*(volatile uint32_t *)&a.ctl->done) return;
    if (threadIdx.x != 0 || blockIdx.x != 0 || a.V == 0) return;
    float b[MS];
    ldv<MS>(a.belief, b);
    for (uint32_t r = 0; r < a.nruns; ++r) {
        const int s = a.run_s[r];
        const uint32_t len = a.run_len[r];
        for (uint32_t k = 0; k < len; ++k) {
            float sum = 0.0f;
#pragma unroll
            for (int i = 0; i < MS; ++i)
                if (i < s) sum = FADD(sum, b[i]);
            if (!(sum > 0.0f)) break;
            bool changed = false;
#pragma unroll
            for (int i = 0; i < MS; ++i) {
                if (i < s) {
                    float nb = FDIV(b[i], sum);
                    changed |= __float_as_uint(nb) != __float_as_uint(b[i]);
                    b[i] = nb;
                }
            }
            if (!changed) break;
        }
    }
    stv<MS>(a.belief, b);
}

template <int MS, bool UNI>
__global__ void __launch_bounds__(256) k_edge_delta(const EdgeArgs a) {
    __shared__ double red[8];
    __shared__ bool s_last;
    __shared__ __align__(16) float buf[2 * 1024];
    LoopyCtl *ctl = a.ctl;
    if (*(volatile uint32_t *)&ctl->done) return;
    const uint32_t it = ctl->it, ce = ctl->check_every;
    const bool want = (ce <= 1) || ((it + 1) % ce == 0);
    const bool serial = ctl->serial != 0;
    float *absd = check_buffer(ctl, a.absdiff, it, want);
    // the delta reads the local prev/curr AFTER this iteration's swap (_acc)
    float *prev, *curr;
    edge_roles(a, ctl->acc_edge ? it + 1 : it, prev, curr);
    double dsum = 0.0;
    const uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (want && p < a.E) {
        int x = MS;
        if (!UNI) x = a.pos_dims[p] & 15;
        float o[MS], c[MS], ad[MS];
        ldv<MS>(prev + p * MS, o);
        ldv<MS>(curr + p * MS, c);
#pragma unroll
        for (int k = 0; k < MS; ++k) {
            float d = 0.0f;
            if (UNI || k < x) {
                d = FSUB(o[k], c[k]);
                if (d != d) d = 0.0f;
                d = fabsf(d);
            }
            ad[k] = d;
            dsum += (double)d;
        }
        if (absd) stv<MS>(absd + (size_t)a.pos_edge[p] * MS, ad);
    }
    if (serial) reduce_and_finalize<256, true>(ctl, a.partials, dsum, want, red, &s_last, a.absdiff, buf, 2 * 1024);
    else reduce_and_finalize<256>(ctl, a.partials, dsum, want, red, &s_last);
}

// ---------------------------------------------------------------- driver --

static int ensure_partials(bp_graph *g, uint32_t n) {
    if (g->partials_cap >= n) return BP_OK;
    if (g->partials) {
        cudaFreeAsync(g->partials, g->stream);
        g->partials = nullptr;
    }
    for (auto &c : g->loop_graph)
        if (c.exec) {
            cudaGraphExecDestroy(c.exec);
            c.exec = nullptr;
            c.key = 0;
        }
    int st = dev_alloc(g, (void **)&g->partials, sizeof(double) * n);
    if (st == BP_OK) g->partials_cap = n;
    return st;
}

// floats between the three |diff| buffers of the serial delta (16-byte
// aligned starts for the serial sum's float4 reads)
static uint64_t absdiff_stride(const bp_graph *g) { return ((uint64_t)g->E * g->ms + 3u) & ~3ull; }

static int ensure_absdiff(bp_graph *g) {
    if (g->absdiff) return BP_OK;
    for (auto &c : g->loop_graph)
        if (c.exec) {
            cudaGraphExecDestroy(c.exec);
            c.exec = nullptr;
            c.key = 0;
        }
    const size_t bytes = sizeof(float) * (3 * (size_t)absdiff_stride(g) + 4);
    int st = dev_alloc(g, (void **)&g->absdiff, bytes);
    if (st) return st;
    BP_CUDA(cudaMemsetAsync(g->absdiff, 0, bytes, g->stream));
    return BP_OK;
}

// runs of equal state count over node order, for the node-0 normalisation
static int ensure_runs(bp_graph *g) {
    if (g->run_len || g->V == 0) return BP_OK;
    std::vector<uint32_t> len;
    std::vector<uint8_t> s;
    for (uint32_t v = 0; v < g->V; ++v) {
        if (s.empty() || s.back() != g->node_s_host[v]) {
            s.push_back(g->node_s_host[v]);
            len.push_back(0);
        }
        len.back()++;
    }
    int st;
    if ((st = dev_alloc(g, (void **)&g->run_len, sizeof(uint32_t) * len.size()))) return st;
    if ((st = dev_alloc(g, (void **)&g->run_s, s.size()))) return st;
    BP_CUDA(cudaMemcpy(g->run_len, len.data(), sizeof(uint32_t) * len.size(), cudaMemcpyHostToDevice));
    BP_CUDA(cudaMemcpy(g->run_s, s.data(), s.size(), cudaMemcpyHostToDevice));
    g->nruns = (uint32_t)len.size();
    return BP_OK;
}

template <int MS, bool UNI>
static int launch_init(bp_graph *g) {
    if (g->E == 0) return BP_OK;
    k_send_from_beliefs<MS, UNI><<<grid_for(g->E, 256), 256, 0, g->stream>>>(g->E, g->in_src, g->pos_dims, g->joint,
                                                                             g->belief, g->msg[g->latest]);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

template <int MS, bool UNI>
static int launch_gather(bp_graph *g) {
    if (g->V == 0) return BP_OK;
    k_gather_q<MS, UNI><<<grid_for(g->V, 256), 256, 0, g->stream>>>(g->V, g->in_ptr, g->node_s, g->belief,
                                                                     g->msg[g->latest], g->q[0]);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

// nodes whose send-buffer entries get the evict-last policy: the renumbered
// nodes with two or more out-edges, at most BP_FLOOD_HOT_MB (default 48) MB
// of send buffer
static uint32_t flood_hot_nodes(const bp_graph *g) {
    size_t mb = 48;
    if (const char *env = getenv("BP_FLOOD_HOT_MB")) mb = (size_t)atol(env);
    const size_t cap = (mb << 20) / (sizeof(float) * g->ms);
    return (uint32_t)std::min<size_t>(g->reuse_nodes, cap);
}

static FloodArgs flood_args(bp_graph *g) {
    FloodArgs a;
    a.V = g->V;
    a.v_base = 0;
    a.hot = flood_hot_nodes(g);
    {
        // default 1: on the 16M-node graph 0.974 -> 0.932 ms per iteration
        // (2 spills registers and is slower); BP_FLOOD_PIPE overrides
        const char *env = getenv("BP_FLOOD_PIPE");
        a.pipe = env ? (uint32_t)atoi(env) : 1u;
    }
    a.in_ptr = g->in_ptr;
    a.in_src = g->in_src;
    a.pos_edge = g->pos_edge;
    a.node_s = g->node_s;
    a.pos_dims = g->pos_dims;
    a.joint = g->joint;
    a.belief = g->belief;
    a.msg0 = g->msg[0];
    a.msg1 = g->msg[1];
    a.q0 = g->q[0];
    a.q1 = g->q[1];
    a.partials = g->partials;
    a.absdiff = g->absdiff;
    a.ctl = g->ctl;
    return a;
}

static EdgeArgs edge_args(bp_graph *g) {
    EdgeArgs a;
    a.V = g->V;
    a.E = g->E;
    a.in_ptr = g->in_ptr;
    a.in_src = g->in_src;
    a.pos_edge = g->pos_edge;
    a.edge_pos = g->edge_pos;
    a.node_s = g->node_s;
    a.pos_dims = g->pos_dims;
    a.joint = g->joint;
    a.belief = g->belief;
    a.msg0 = g->msg[0];
    a.msg1 = g->msg[1];
    a.partials = g->partials;
    a.absdiff = g->absdiff;
    a.ctl = g->ctl;
    a.run_len = g->run_len;
    a.run_s = g->run_s;
    a.nruns = g->nruns;
    return a;
}

// staged kernel: dynamic shared memory opt-in (once per process) and the
// persistent grid (resident CTAs per SM x SMs, at most one CTA per tile)
template <int MS>
static int staged_grid(const bp_graph *g, unsigned *grid, uint32_t *ntiles) {
    using C = Staged<MS>;
    static int bps = 0;
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (bps == 0) {
            BP_CUDA(cudaFuncSetAttribute(k_flood_staged<MS>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
            BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_flood_staged<MS>, C::TN, C::SMEM));
            if (bps < 1) return set_error(BP_ERR_CUDA, "staged iteration kernel does not fit an SM");
        }
    }
    int dev = 0, sms = 0;
    BP_CUDA(cudaGetDevice(&dev));
    BP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    *ntiles = (g->V + C::TN - 1) / C::TN;
    *grid = (unsigned)std::min<uint64_t>(*ntiles, (uint64_t)bps * sms);
    return BP_OK;
}

// edges in flight per thread of the block-tile kernel: BP_FLOOD_UNROLL=1|2|4
// overrides the default for 1- and 2-state graphs (every choice gives the
// same results)
template <int MS>
static int block_unroll() {
    int unroll = flood_unroll<MS>();
    if constexpr (MS <= 2) {
        const char *env = getenv("BP_FLOOD_UNROLL");
        if (env && (env[0] == '1' || env[0] == '2' || env[0] == '4')) unroll = env[0] - '0';
    }
    return unroll;
}

// resident blocks per SM the block-tile kernel's registers are capped for:
// BP_FLOOD_MINB=10|16 overrides flood_min_blocks (12) for 1- and 2-state
// graphs (resident 128-thread blocks per SM), for sweeps; 0 = the default
static int block_min_blocks() {
    const char *env = getenv("BP_FLOOD_MINB");
    const int v = env ? atoi(env) : 0;
    return (v == 10 || v == 16) ? v : 0;
}

template <int MS, bool UNI, int FU, int MB>
static int resident_blocks_mb(int *bps) {
    static int cached = 0;
    if (!cached)
        BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cached, k_flood<MS, UNI, FU, MB>, flood_nt<MS>(), 0));
    *bps = cached;
    return BP_OK;
}

template <int MS, bool UNI, int FU>
static int resident_blocks(int *bps) {
    if constexpr (MS <= 2) {
        const int mb = block_min_blocks();
        if (mb == 10) return resident_blocks_mb<MS, UNI, FU, 10>(bps);
        if (mb == 16) return resident_blocks_mb<MS, UNI, FU, 16>(bps);
    }
    return resident_blocks_mb<MS, UNI, FU, flood_min_blocks<MS, FU>()>(bps);
}

// launch of the block-tile kernel with the register cap block_min_blocks()
template <int MS, bool UNI, int FU>
static void launch_block_tiles(unsigned grid, cudaStream_t st, const FloodArgs &a, uint32_t ntiles, bool serial) {
    constexpr int NT = flood_nt<MS>();
    constexpr int MB = flood_min_blocks<MS, FU>();
    if (serial) return k_flood<MS, UNI, FU, MB, true><<<grid, NT, 0, st>>>(a, ntiles);
    if constexpr (MS <= 2) {
        const int mb = block_min_blocks();
        if (mb == 10) return k_flood<MS, UNI, FU, 10><<<grid, NT, 0, st>>>(a, ntiles);
        if (mb == 16) return k_flood<MS, UNI, FU, 16><<<grid, NT, 0, st>>>(a, ntiles);
    }
    k_flood<MS, UNI, FU><<<grid, NT, 0, st>>>(a, ntiles);
}

// block-tile grid: one block per tile, or (default; BP_FLOOD_PERSIST=0
// turns it off) a persistent grid of resident blocks x SMs walking the tiles
template <int MS, bool UNI>
static int block_tiles(const bp_graph *g, unsigned *grid, uint32_t *ntiles) {
    *ntiles = grid_for(g->V, flood_nt<MS>());
    *grid = *ntiles;
    const char *env = getenv("BP_FLOOD_PERSIST");
    if (env && env[0] == '0') return BP_OK;
    int bps = 0, st;
    if constexpr (MS <= 2) {
        const int fu = block_unroll<MS>();
        st = fu == 1 ? resident_blocks<MS, UNI, 1>(&bps)
                     : (fu == 2 ? resident_blocks<MS, UNI, 2>(&bps) : resident_blocks<MS, UNI, 4>(&bps));
    } else {
        st = resident_blocks<MS, UNI, flood_unroll<MS>()>(&bps);
    }
    if (st) return st;
    int dev = 0, sms = 0;
    BP_CUDA(cudaGetDevice(&dev));
    BP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (bps > 0) *grid = (unsigned)std::min<uint64_t>(*ntiles, (uint64_t)bps * sms);
    return BP_OK;
}

// ---- the split schedule (flood_split.cuh) ----------------------------------

// send buffers per source range: BP_FLOOD_RANGE_MB (default 32) MB, or
// BP_FLOOD_RANGE_NODES nodes
static uint32_t split_range_nodes(const bp_graph *g) {
    if (const char *env = getenv("BP_FLOOD_RANGE_NODES")) return std::max<uint32_t>(1, (uint32_t)atol(env));
    size_t mb = 32;
    if (const char *env = getenv("BP_FLOOD_RANGE_MB")) mb = std::max<size_t>(1, (size_t)atol(env));
    const uint64_t rn = std::max<uint64_t>(1, (mb << 20) / (sizeof(float) * g->ms));
    return (uint32_t)std::min<uint64_t>(rn, 0xffffffffu);
}

// BP_FLOOD_SPLIT=1: whenever the layout applies; =0: never; default (auto):
// when the send buffers exceed BP_FLOOD_SPLIT_MIN_MB (default 64) MB, i.e.
// when they no longer stay in L2 across an iteration.  On the 16.8M-node
// power-law graph (nodes renumbered, in-degree tie-break) the split loop cuts
// DRAM traffic from 4.8 to 3.85 GB per iteration and runs 0.755-0.78 ms
// against k_flood's 0.85-0.88 ms; its layout (a second edge order: a radix
// sort and a 2.7 GB gather) adds about 2 ms of host time and 14 ms of device
// work to a graph build, which a serving loop overlaps with the previous
// solve (101 against 106 ms per build + 100-iteration solve).
static bool split_wanted(const bp_graph *g) {
    const char *env = getenv("BP_FLOOD_SPLIT");
    if (env && env[0] == '0') return false;
    if (env && env[0] == '1') return true;
    size_t mb = 64;
    if (const char *e2 = getenv("BP_FLOOD_SPLIT_MIN_MB")) mb = (size_t)atol(e2);
    return (uint64_t)g->V * g->ms * sizeof(float) > ((uint64_t)mb << 20);
}

static int split_prepare(bp_graph *g) { return split_build(g, split_range_nodes(g)); }

// build the split layout of a graph the default loop would run it on (the
// graph build calls this, so a serving loop's next graph is prepared beside
// the current solve); a no-op for graphs it does not apply to
int flood_split_prepare(bp_graph *g) {
    if (g->split.state || !g->uniform || g->ms > 4 || g->E == 0 || !split_wanted(g)) return BP_OK;
    return split_prepare(g);
}

static SplitArgs split_args(bp_graph *g, uint32_t nparts) {
    SplitArgs a;
    const auto &s = g->split;
    a.V = g->V;
    a.E = g->E;
    a.in_ptr = g->in_ptr;
    a.s_src = s.s_src;
    a.s_edge = s.s_edge;
    a.s_inv = s.s_inv;
    a.s_joint = s.s_joint;
    a.s_msg0 = s.s_msg[0];
    a.s_msg1 = s.s_msg[1];
    a.q0 = g->q[0];
    a.q1 = g->q[1];
    a.belief = g->belief;
    a.partials = g->partials;
    a.nparts = nparts;
    a.absdiff = g->absdiff;
    a.ctl = g->ctl;
    return a;
}

// k launches of (send pass, node pass), or (k == 0) the send pass's block
// count only (the delta partials it writes): resident blocks x SMs, at most
// one block per 256 edges
template <int MS, bool SER, int NV>
static int split_run_nv(bp_graph *g, uint32_t k, uint32_t *nparts) {
    static int bps_a = 0, bps_b = 0;
    static std::mutex mu;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (bps_a == 0) {
            BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_a, k_flood_send<MS, SER>, kSendThreads, 0));
            BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps_b, k_flood_nodes<MS, SER, NV>,
                                                                  kNodeThreads, 0));
            if (bps_a < 1 || bps_b < 1) return set_error(BP_ERR_CUDA, "split iteration kernels do not fit an SM");
        }
    }
    int dev = 0, sms = 0;
    BP_CUDA(cudaGetDevice(&dev));
    BP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned ga = std::min<unsigned>((unsigned)(bps_a * sms), grid_for(g->E, kSendThreads));
    const unsigned gb = std::min<unsigned>((unsigned)(bps_b * sms), grid_for(g->V, kNodeThreads));
    if (nparts) *nparts = ga;
    const SplitArgs a = split_args(g, ga);
    for (uint32_t i = 0; i < k; ++i) {
        k_flood_send<MS, SER><<<ga, kSendThreads, 0, g->stream>>>(a);
        k_flood_nodes<MS, SER, NV><<<gb, kNodeThreads, 0, g->stream>>>(a);
        BP_CUDA(cudaGetLastError());
    }
    return BP_OK;
}

// BP_SPLIT_NODES=0|1|2|3: the node pass's load form (sweeps, 2-state
// graphs).  3, the default, loads the next node's row pointers and belief one
// round ahead (32 registers, every thread slot of an SM): 0.767 ms per
// iteration on the 16.8M-node graph against 0.782 for 1 (the compiler-
// unrolled loop alone); with ties broken by id, forms 0-2 measured 0.876,
// 0.859 and 0.864 ms; a group of 4 lanes per node, each lane repeating the
// node's products, measured 2.06 ms and was removed.
template <int MS, bool SER>
static int split_run(bp_graph *g, uint32_t k, uint32_t *nparts) {
    if constexpr (MS == 2) {
        const char *env = getenv("BP_SPLIT_NODES");
        const int nv = env ? atoi(env) : 3;
        if (nv == 0) return split_run_nv<MS, SER, 0>(g, k, nparts);
        if (nv == 2) return split_run_nv<MS, SER, 2>(g, k, nparts);
        if (nv == 1) return split_run_nv<MS, SER, 1>(g, k, nparts);
    }
    return split_run_nv<MS, SER, 3>(g, k, nparts);
}

template <int MS, bool UNI>
static int enqueue_split_iterations(bp_graph *g, uint32_t k, bool serial) {
    if constexpr (!UNI || MS > 4) {
        return set_error(BP_ERR_INVALID, "split schedule: uniform graphs of at most 4 states");
    } else {
        return serial ? split_run<MS, true>(g, k, nullptr) : split_run<MS, false>(g, k, nullptr);
    }
}

// the send pass's grid (the delta partials it writes)
template <int MS, bool UNI>
static int split_send_blocks(bp_graph *g, bool serial, uint32_t *n) {
    if constexpr (!UNI || MS > 4) {
        return set_error(BP_ERR_INVALID, "split schedule: uniform graphs of at most 4 states");
    } else {
        return serial ? split_run<MS, true>(g, 0, n) : split_run<MS, false>(g, 0, n);
    }
}

// messages between position order and send order (dir 0: the latest slot
// into send order; dir 1: both slots back)
template <int MS, bool UNI>
static int split_convert(bp_graph *g, int dir) {
    if constexpr (!UNI || MS > 4) {
        return set_error(BP_ERR_INVALID, "split schedule: uniform graphs of at most 4 states");
    } else {
        const auto &s = g->split;
        if (dir == 0) {
            k_to_send_order<MS><<<grid_for(g->E, 256), 256, 0, g->stream>>>(s.s_pos, g->E, g->msg[g->latest],
                                                                             s.s_msg[g->latest]);
        } else {
            for (int k = 0; k < 2; ++k)
                k_from_send_order<MS><<<grid_for(g->E, 256), 256, 0, g->stream>>>(s.s_pos, g->E, s.s_msg[k],
                                                                                  g->msg[k]);
        }
        BP_CUDA(cudaGetLastError());
        return BP_OK;
    }
}

// whether the node schedule's loop runs split (*use): uniform graphs of at
// most 4 states, the default loop (kernel variant AUTO: when split_wanted) or
// BP_KERNEL_SPLIT asked for; the layout is built here if the graph build did
// not; a graph whose node tiles hold too many in-edges keeps k_flood
static int split_applies(bp_graph *g, int schedule, int variant, bool *use) {
    *use = false;
    if (schedule != BP_SCHEDULE_NODE || !g->uniform || g->ms > 4 || g->E == 0 || g->V == 0) return BP_OK;
    if (variant != BP_KERNEL_AUTO && variant != BP_KERNEL_SPLIT) return BP_OK;
    if (variant == BP_KERNEL_AUTO && !split_wanted(g)) return BP_OK;
    if (g->split.state == 0) {
        int st = split_prepare(g);
        if (st) return st;
    }
    *use = g->split.state == 1;
    return BP_OK;
}

template <int MS, bool UNI>
static int enqueue_node_iterations(bp_graph *g, uint32_t k, bool serial, int variant) {
    constexpr int NT = flood_nt<MS>();
    if (variant == BP_KERNEL_STAGED_TILE) {
        if constexpr (UNI && MS == 2) {
            unsigned grid = 0;
            uint32_t ntiles = 0;
            int st = staged_grid<MS>(g, &grid, &ntiles);
            if (st) return st;
            const FloodArgs a = flood_args(g);
            for (uint32_t i = 0; i < k; ++i) {
                k_flood_staged<MS><<<grid, Staged<MS>::TN, Staged<MS>::SMEM, g->stream>>>(a, ntiles);
                BP_CUDA(cudaGetLastError());
            }
            return BP_OK;
        } else {
            return set_error(BP_ERR_INVALID, "staged tiles need a uniform 2-state graph");
        }
    }
    const bool warp_tiled = variant != BP_KERNEL_BLOCK_TILE;
    unsigned grid = grid_for(g->V, 256);
    uint32_t ntiles = 0;
    if (!warp_tiled) {
        int st = block_tiles<MS, UNI>(g, &grid, &ntiles);
        if (st) return st;
    }
    const FloodArgs a = flood_args(g);
    const int unroll = warp_tiled ? wflood_unroll<MS>() : block_unroll<MS>();
    for (uint32_t i = 0; i < k; ++i) {
        if (!warp_tiled) {
            if constexpr (MS <= 2) {
                if (unroll == 1) launch_block_tiles<MS, UNI, 1>(grid, g->stream, a, ntiles, serial);
                else if (unroll == 2) launch_block_tiles<MS, UNI, 2>(grid, g->stream, a, ntiles, serial);
                else launch_block_tiles<MS, UNI, 4>(grid, g->stream, a, ntiles, serial);
            } else {
                constexpr int FU = flood_unroll<MS>();
                if (serial) k_flood<MS, UNI, FU, flood_min_blocks<MS, FU>(), true><<<grid, NT, 0, g->stream>>>(a, ntiles);
                else k_flood<MS, UNI, FU><<<grid, NT, 0, g->stream>>>(a, ntiles);
            }
        } else if constexpr (MS <= 2) {
            if (unroll == 1) k_flood_w<MS, UNI, 1><<<grid, 256, 0, g->stream>>>(a);
            else if (unroll == 2) k_flood_w<MS, UNI, 2><<<grid, 256, 0, g->stream>>>(a);
            else k_flood_w<MS, UNI, 4><<<grid, 256, 0, g->stream>>>(a);
        } else {
            k_flood_w<MS, UNI, wflood_unroll<MS>()><<<grid, 256, 0, g->stream>>>(a);
        }
        BP_CUDA(cudaGetLastError());
    }
    return BP_OK;
}

template <int MS, bool UNI>
static int enqueue_edge_iterations(bp_graph *g, uint32_t k, bool, int) {
    const EdgeArgs a = edge_args(g);
    const uint64_t n = (uint64_t)g->E * MS;
    for (uint32_t i = 0; i < k; ++i) {
        k_edge_copy<MS><<<grid_for(n, 256), 256, 0, g->stream>>>(a);
        k_edge_send<MS, UNI><<<grid_for(g->E, 256), 256, 0, g->stream>>>(a);
        k_edge_combine<MS, UNI><<<grid_for(g->V, 256), 256, 0, g->stream>>>(a);
        k_edge_normalise_node0<MS><<<1, 32, 0, g->stream>>>(a);
        k_edge_delta<MS, UNI><<<grid_for(g->E, 256), 256, 0, g->stream>>>(a);
        BP_CUDA(cudaGetLastError());
    }
    return BP_OK;
}

static int enqueue_iterations(bp_graph *g, int schedule, uint32_t k, bool serial, int variant) {
    if (schedule == BP_SCHEDULE_NODE && variant == BP_KERNEL_SPLIT)
        BP_DISPATCH_MS(g->ms, g->uniform != 0, enqueue_split_iterations, g, k, serial);
    if (schedule == BP_SCHEDULE_NODE)
        BP_DISPATCH_MS(g->ms, g->uniform != 0, enqueue_node_iterations, g, k, serial, variant);
    BP_DISPATCH_MS(g->ms, g->uniform != 0, enqueue_edge_iterations, g, k, serial, variant);
}

static int flood_grid(bp_graph *g, int variant, uint32_t *grid, bool serial) {
    if (variant == BP_KERNEL_SPLIT) {
        auto f = [&]() -> int { BP_DISPATCH_MS(g->ms, g->uniform != 0, split_send_blocks, g, serial, grid); };
        return f();
    }
    if (variant == BP_KERNEL_STAGED_TILE) {
        uint32_t ntiles = 0;
        unsigned gr = 0;
        int st = staged_grid<2>(g, &gr, &ntiles);
        *grid = gr;
        return st;
    }
    if (variant == BP_KERNEL_BLOCK_TILE) {
        uint32_t ntiles = 0;
        auto tiles = [&]() -> int { BP_DISPATCH_MS(g->ms, g->uniform != 0, block_tiles, g, grid, &ntiles); };
        return tiles();
    }
    *grid = grid_for(g->V, 256);
    return BP_OK;
}

// the staged kernel applies to uniform 2-state graphs on the node schedule
// with the f64 delta, whose arrays are 16-byte aligned and whose mean
// in-degree leaves the typical tile inside a stage (<= 3/4 of CAP edges)
static bool staged_applies(const bp_graph *g, int schedule, bool serial) {
    if (schedule != BP_SCHEDULE_NODE || serial || g->uniform != 2) return false;
    if ((uint64_t)g->E * Staged<2>::TN > (uint64_t)g->V * (Staged<2>::CAP * 3 / 4)) return false;
    const uintptr_t any = (uintptr_t)g->in_ptr | (uintptr_t)g->in_src | (uintptr_t)g->joint |
                          (uintptr_t)g->belief | (uintptr_t)g->msg[0] | (uintptr_t)g->msg[1];
    return (any & 15u) == 0;
}

// the fused loop: its grid (at most one co-resident block per tile), or 0
// when the graph has more tiles than the GPU holds blocks at once
template <int MS, bool UNI>
static int fused_grid(const bp_graph *g, unsigned *grid, uint32_t *ntiles, bool serial) {
    constexpr int FU = flood_unroll<MS>();
    static int bps_f64 = -1, bps_ser = -1;
    int &bps = serial ? bps_ser : bps_f64;
    if (bps < 0) {
        if (serial)
            BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_flood_fused<MS, UNI, FU, true>,
                                                                  flood_nt<MS>(), 0));
        else
            BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_flood_fused<MS, UNI, FU>, flood_nt<MS>(), 0));
    }
    int dev = 0, sms = 0;
    BP_CUDA(cudaGetDevice(&dev));
    BP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    *ntiles = grid_for(g->V, flood_nt<MS>());
    *grid = (bps > 0 && (uint64_t)*ntiles <= (uint64_t)bps * sms) ? *ntiles : 0u;
    return BP_OK;
}

template <int MS, bool UNI>
static int launch_fused(bp_graph *g, unsigned grid, uint32_t ntiles, bool serial) {
    constexpr int FU = flood_unroll<MS>();
    FloodArgs a = flood_args(g);
    void *args[] = {(void *)&a, (void *)&ntiles};
    const void *fn = serial ? (const void *)k_flood_fused<MS, UNI, FU, true> : (const void *)k_flood_fused<MS, UNI, FU>;
    BP_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(flood_nt<MS>()), args, 0, g->stream));
    return BP_OK;
}

// ---- one rank's node range of a sharded run ----------------------------

template <int MS, bool UNI>
static int launch_gather_range(bp_graph *g, uint32_t v0, uint32_t v1, float *q_out, cudaStream_t st) {
    if (v1 > v0)
        k_gather_q<MS, UNI><<<grid_for(v1 - v0, 256), 256, 0, st>>>(v1 - v0, g->in_ptr + v0, g->node_s + v0,
                                                                    g->belief + (size_t)v0 * MS, g->msg[g->latest],
                                                                    q_out + (size_t)v0 * MS);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

template <int MS, bool UNI>
static int launch_flood_range(bp_graph *g, uint32_t v0, uint32_t v1, const float *q_in, float *q_out,
                              double *delta, cudaStream_t st) {
    constexpr int NT = flood_nt<MS>();
    constexpr int FU = flood_unroll<MS>();
    static int bps = 0;
    if (!bps) BP_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_flood_range<MS, UNI, FU>, NT, 0));
    int dev = 0, sms = 0;
    BP_CUDA(cudaGetDevice(&dev));
    BP_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t ntiles = (v1 - v0 + NT - 1) / NT;
    const uint32_t grid = std::min<uint32_t>(ntiles, (uint32_t)std::max(1, bps * sms));
    int rc;
    if ((rc = ensure_partials(g, std::max(grid, 1u)))) return rc;
    FloodArgs a = flood_args(g);
    a.V = v1;
    a.v_base = v0;
    a.hot = 0;
    if (ntiles)
        k_flood_range<MS, UNI, FU><<<grid, NT, 0, st>>>(a, ntiles, g->msg[g->latest], g->msg[g->latest ^ 1], q_in,
                                                        q_out, g->partials);
    k_sum_partials<<<1, 256, 0, st>>>(g->partials, ntiles ? grid : 0u, delta);
    BP_CUDA(cudaGetLastError());
    g->latest ^= 1;
    return BP_OK;
}

static int range_check(const bp_graph *g, uint32_t v0, uint32_t v1) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    if (v0 > v1 || v1 > g->V) return set_error(BP_ERR_INVALID, "node range [%u, %u) not inside [0, %u)", v0, v1, g->V);
    if (g->new_to_old)
        return set_error(BP_ERR_STATE, "node ranges of a renumbered graph (BP_GRAPH_REORDER_BY_OUT_DEGREE)");
    return BP_OK;
}

}  // namespace bpx

using namespace bpx;

extern "C" {

int bp_send_buffers_range(bp_graph *g, uint32_t node_begin, uint32_t node_end, float *q_out, void *stream) {
    int st = range_check(g, node_begin, node_end);
    if (st) return st;
    if (!q_out) return set_error(BP_ERR_INVALID, "null send buffers");
    cudaStream_t s = stream ? (cudaStream_t)stream : g->stream;
    BP_DISPATCH_MS(g->ms, g->uniform != 0, launch_gather_range, g, node_begin, node_end, q_out, s);
}

int bp_flood_range(bp_graph *g, uint32_t node_begin, uint32_t node_end, const float *q_in, float *q_out,
                   double *delta, void *stream) {
    NvtxRange nvtx("bp_flood_range");
    int st = range_check(g, node_begin, node_end);
    if (st) return st;
    if (!q_in || !q_out || !delta) return set_error(BP_ERR_INVALID, "null argument");
    if (q_in == q_out) return set_error(BP_ERR_INVALID, "q_in and q_out must be different buffers");
    cudaStream_t s = stream ? (cudaStream_t)stream : g->stream;
    BP_DISPATCH_MS(g->ms, g->uniform != 0, launch_flood_range, g, node_begin, node_end, q_in, q_out, delta, s);
}

void bp_loopy_default_options(bp_loopy_options *o) {
    if (!o) return;
    o->tolerance = 1e-3f;
    o->max_iterations = 200;
    o->check_every = 1;
    o->schedule = BP_SCHEDULE_NODE;
    o->delta_mode = BP_DELTA_AUTO;
    o->verbose = 0;
    o->graph_chunk = 0;
    o->kernel_variant = BP_KERNEL_AUTO;
}

int bp_init_messages(bp_graph *g) {
    if (!g) return set_error(BP_ERR_INVALID, "null graph");
    BP_DISPATCH_MS(g->ms, g->uniform != 0, launch_init, g);
}

int bp_serial_sum_bounds(const float *x, uint64_t n, double *lohi, void *stream) {
    if (!lohi || (n && !x)) return set_error(BP_ERR_INVALID, "null argument");
    k_serial_sum_bounds<<<1, 256, 0, (cudaStream_t)stream>>>(x, n, lohi);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

int bp_serial_sum_f32(const float *x, uint64_t n, float *out, int method, void *stream) {
    if (!out || (n && !x)) return set_error(BP_ERR_INVALID, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    switch (method) {
    case 0: k_serial_sum<256><<<1, 256, 0, st>>>(x, n, out, 0, 8192); break;
    case 1: k_serial_sum<128><<<1, 128, 0, st>>>(x, n, out, 0, 2048); break;
    case 2: k_serial_sum<256><<<1, 256, 0, st>>>(x, n, out, 0, 2048); break;
    case 3: k_serial_sum<256><<<1, 256, 0, st>>>(x, n, out, 1, 8192); break;
    case 4: k_serial_sum<1024><<<1, 1024, 0, st>>>(x, n, out, 0, 8192); break;
    default: return set_error(BP_ERR_INVALID, "unknown method %d", method);
    }
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

int bp_loopy(bp_graph *g, const bp_loopy_options *opt, bp_loopy_result *res) {
    NvtxRange nvtx("bp_loopy");
    if (!g || !opt) return set_error(BP_ERR_INVALID, "null argument");
    if (opt->schedule != BP_SCHEDULE_NODE && opt->schedule != BP_SCHEDULE_EDGE)
        return set_error(BP_ERR_INVALID, "unknown schedule %d", opt->schedule);
    if (opt->delta_mode < BP_DELTA_AUTO || opt->delta_mode > BP_DELTA_F64)
        return set_error(BP_ERR_INVALID, "unknown delta mode %d", opt->delta_mode);
    if (opt->schedule == BP_SCHEDULE_EDGE && g->new_to_old)
        return set_error(BP_ERR_STATE, "edge schedule on a renumbered graph (BP_GRAPH_REORDER_BY_OUT_DEGREE)");
    const uint32_t ce = opt->check_every <= 1 ? 1u : opt->check_every;
    const uint32_t max_it = opt->max_iterations;
    bp_loopy_result r = {};
    r.previous_delta = -1.0f;
    const bool serial = opt->delta_mode == BP_DELTA_SERIAL_F32 ||
                        (opt->delta_mode == BP_DELTA_AUTO && (uint64_t)g->E * g->ms <= (1ull << 20));
    // degenerate loops: nothing launches (the reference's loop body never
    // runs, or there is no node to hold a delta)
    if (max_it == 0 || g->V == 0) {
        float prev = -1.0f, delta = 0.0f;
        uint32_t i = 0, executed = 0, num_iter = 0;
        if (ce <= 1) {
            for (i = 0; i < max_it; ++i) {
                ++executed;
                delta = 0.0f;
                if (delta < opt->tolerance || fabsf(delta - prev) < opt->tolerance) break;
                if (i < max_it - 1) prev = delta;
            }
            r.iterations = i;
        } else {
            for (i = 0; i < max_it; i += ce) {
                executed += ce;
                delta = 0.0f;
                if (delta < opt->tolerance || fabsf(delta - prev) < opt->tolerance) break;
                prev = delta;
                num_iter += ce;
            }
            r.iterations = num_iter;
        }
        r.executed = executed;
        r.converged = i < max_it;
        r.delta = delta;
        r.previous_delta = prev;
        r.delta_f64 = delta;
        if (i == max_it && opt->verbose)
            printf("No Convergence: previous: %f vs current: %f\n", (double)prev, (double)delta);
        if (opt->schedule == BP_SCHEDULE_NODE && ce <= 1 && (executed & 1u)) g->latest ^= 1;
        if (res) *res = r;
        return BP_OK;
    }
    int st;
    int variant = opt->kernel_variant;
    if (variant == BP_KERNEL_SPLIT) variant = BP_KERNEL_BLOCK_TILE;   // resolved below
    if (variant == BP_KERNEL_AUTO) {
        const char *env = getenv("BP_FLOOD_KERNEL");
        if (env && env[0] == 'w') variant = BP_KERNEL_WARP_TILE;
        else if (env && env[0] == 's' && staged_applies(g, opt->schedule, serial)) variant = BP_KERNEL_STAGED_TILE;
        else variant = BP_KERNEL_BLOCK_TILE;
    }
    if (variant == BP_KERNEL_BLOCK_TILE && (opt->kernel_variant == BP_KERNEL_AUTO || opt->kernel_variant == BP_KERNEL_SPLIT)) {
        // large uniform graphs: the split schedule (send pass in source-range
        // order + node pass)
        bool use = false;
        if ((st = split_applies(g, opt->schedule, opt->kernel_variant, &use))) return st;
        if (use) variant = BP_KERNEL_SPLIT;
        else if (opt->kernel_variant == BP_KERNEL_SPLIT)
            return set_error(BP_ERR_INVALID, "split tiles need the node schedule on a uniform graph of at most 4 "
                                             "states");
    }
    if (variant != BP_KERNEL_BLOCK_TILE && variant != BP_KERNEL_WARP_TILE && variant != BP_KERNEL_STAGED_TILE &&
        variant != BP_KERNEL_SPLIT)
        return set_error(BP_ERR_INVALID, "unknown kernel variant %d", opt->kernel_variant);
    if (variant == BP_KERNEL_STAGED_TILE && opt->schedule == BP_SCHEDULE_NODE && !staged_applies(g, opt->schedule, serial))
        return set_error(BP_ERR_INVALID, "staged tiles need a uniform 2-state graph of mean in-degree <= 4.5 and the f64 delta");
    uint32_t grid_blocks = grid_for(g->E, 256);
    if (opt->schedule == BP_SCHEDULE_NODE && (st = flood_grid(g, variant, &grid_blocks, serial))) return st;
    // small graphs (a co-resident block per tile), node schedule, f64 delta,
    // block tiles: every iteration in one cooperative launch
    // (BP_FLOOD_FUSED=0 keeps the launch-per-iteration loop)
    unsigned fgrid = 0;
    uint32_t fntiles = 0;
    {
        const char *env = getenv("BP_FLOOD_FUSED");
        if (opt->schedule == BP_SCHEDULE_NODE && variant == BP_KERNEL_BLOCK_TILE &&
            !(env && env[0] == '0')) {
            auto fg = [&]() -> int { BP_DISPATCH_MS(g->ms, g->uniform != 0, fused_grid, g, &fgrid, &fntiles, serial); };
            if ((st = fg())) return st;
        }
    }
    // double-buffered partials, and in serial mode 8 more per block for the
    // grid-wide narrowing
    if (fgrid) grid_blocks = std::max(grid_blocks, (serial ? 10u : 2u) * fgrid);
    if ((st = ensure_partials(g, grid_blocks))) return st;
    if (serial && (st = ensure_absdiff(g))) return st;
    if (opt->schedule == BP_SCHEDULE_EDGE && ((st = ensure_runs(g)) || (st = ensure_edge_pos(g)))) return st;

    const uint32_t n_launch = ce <= 1 ? max_it : ((max_it + ce - 1) / ce) * ce;
    uint32_t chunk = opt->graph_chunk;
    if (chunk == 0) chunk = opt->schedule == BP_SCHEDULE_NODE ? 32 : 8;
    if (chunk > n_launch) chunk = n_launch;

    LoopyCtl c = {};
    c.max_it = max_it;
    c.check_every = ce;
    c.msg_parity0 = (uint32_t)g->latest;
    c.q_parity0 = 0;
    c.serial = serial ? 1u : 0u;
    c.acc_edge = (opt->schedule == BP_SCHEDULE_EDGE && ce > 1) ? 1u : 0u;
    c.tol = opt->tolerance;
    c.prev_f = -1.0f;
    c.prev_d = -1.0;
    c.n_terms = (uint64_t)g->E * g->ms;
    c.ad_stride = serial ? absdiff_stride(g) : 0;
    c.plo = c.phi = -1.0;
    c.prev_exact = 1;
    c.delta_exact = 1;
    // test hook of the one-launch loop's bounded grid barrier: a shorter
    // wait limit, and a block that does not arrive at the first barrier
    if (const char *env = getenv("BP_DEBUG_WAIT_MS")) c.wait_ms = (uint32_t)strtoul(env, nullptr, 10);
    if (const char *env = getenv("BP_DEBUG_BARRIER_SKIP")) c.bar_skip = (uint32_t)strtoul(env, nullptr, 10) + 1u;
    *g->ctl_host = c;
    BP_CUDA(cudaMemcpyAsync(g->ctl, g->ctl_host, sizeof(LoopyCtl), cudaMemcpyHostToDevice, g->stream));
    if (opt->schedule == BP_SCHEDULE_NODE) {
        auto gather = [&]() -> int { BP_DISPATCH_MS(g->ms, g->uniform != 0, launch_gather, g); };
        if ((st = gather())) return st;
    }
    if (variant == BP_KERNEL_SPLIT) {
        auto conv = [&]() -> int { BP_DISPATCH_MS(g->ms, g->uniform != 0, split_convert, g, 0); };
        if ((st = conv())) return st;
    }

    if (fgrid) {
        BP_CUDA(cudaEventRecord(g->ev0, g->stream));
        auto lf = [&]() -> int { BP_DISPATCH_MS(g->ms, g->uniform != 0, launch_fused, g, fgrid, fntiles, serial); };
        if ((st = lf())) return st;
    } else {
        // CUDA graph of `chunk` iterations, cached per (schedule, delta, chunk)
        const uint64_t key = 1ull | ((uint64_t)opt->schedule << 1) | ((uint64_t)serial << 2) |
                             ((uint64_t)variant << 4) | ((uint64_t)chunk << 8);
        bp_graph::CachedGraph *slot = nullptr;
        for (auto &cg : g->loop_graph)
            if (cg.exec && cg.key == key) slot = &cg;
        if (!slot) {
            slot = &g->loop_graph[0];
            for (auto &cg : g->loop_graph)
                if (!cg.exec) {
                    slot = &cg;
                    break;
                }
            if (slot->exec) {
                cudaGraphExecDestroy(slot->exec);
                slot->exec = nullptr;
            }
            cudaGraph_t graph = nullptr;
            BP_CUDA(cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeThreadLocal));
            st = enqueue_iterations(g, opt->schedule, chunk, serial, variant);
            cudaError_t ce2 = cudaStreamEndCapture(g->stream, &graph);
            if (st) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            if (ce2 != cudaSuccess) return cuda_fail(ce2, "cudaStreamEndCapture", __FILE__, __LINE__);
            cudaError_t ie = cudaGraphInstantiate(&slot->exec, graph, 0);
            cudaGraphDestroy(graph);
            if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
            slot->key = key;
        }

        BP_CUDA(cudaEventRecord(g->ev0, g->stream));
        for (uint32_t launched = 0; launched < n_launch; launched += chunk) {
            BP_CUDA(cudaGraphLaunch(slot->exec, g->stream));
            if (launched + chunk < n_launch) {
                BP_CUDA(cudaMemcpyAsync(&g->ctl_host->done, &g->ctl->done, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                                        g->stream));
                BP_CUDA(cudaStreamSynchronize(g->stream));
                if (g->ctl_host->done) break;
            }
        }
    }
    if (serial) {
        // the returned delta and previous delta where the loop decided
        // without forming them
        k_delta_final<<<2, 1024, 0, g->stream>>>(g->ctl, g->absdiff);
        BP_CUDA(cudaGetLastError());
    }
    BP_CUDA(cudaEventRecord(g->ev1, g->stream));
    if (variant == BP_KERNEL_SPLIT) {
        // both message arrays back to position order (every run executes at
        // least one iteration, so both send-order arrays are defined)
        auto conv = [&]() -> int { BP_DISPATCH_MS(g->ms, g->uniform != 0, split_convert, g, 1); };
        if ((st = conv())) return st;
    }
    BP_CUDA(cudaMemcpyAsync(g->ctl_host, g->ctl, sizeof(LoopyCtl), cudaMemcpyDeviceToHost, g->stream));
    BP_CUDA(cudaStreamSynchronize(g->stream));
    c = *g->ctl_host;
    if (c.done == 3 || c.bar_fail)
        return set_error(BP_ERR_TIMEOUT, "a bounded device wait of the iteration kernel timed out");
    if (!c.done) return set_error(BP_ERR_STATE, "loop ended without a stop decision (it=%u)", c.it);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, g->ev0, g->ev1);
    r.iterations = c.ret;
    r.executed = c.it;
    r.converged = c.done == 1;
    r.delta = serial ? c.delta_f : (float)c.delta_d;
    r.previous_delta = serial ? c.prev_f : (float)c.prev_d;
    r.delta_f64 = c.delta_d;
    r.elapsed_ms = ms;
    r.serial_sums = c.serial_sums;
    r.serial_refines = c.serial_refines;
    r.kernel_used = opt->schedule == BP_SCHEDULE_NODE ? (fgrid ? (int32_t)BP_KERNEL_BLOCK_TILE : (int32_t)variant) : 0;
    if (opt->schedule == BP_SCHEDULE_NODE) g->latest = (int)((c.msg_parity0 + c.it) & 1u);
    if (c.done == 2 && c.final_i == max_it && opt->verbose)
        printf("No Convergence: previous: %f vs current: %f\n", (double)r.previous_delta, (double)r.delta);
    if (res) *res = r;
    return BP_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free loopy BP (bp_loopy_noalloc).
//
// Some callers cannot allocate device memory at the moment they need an
// answer: a host application that owns the GPU's memory through its own
// allocator and forbids other components from calling cudaMalloc, a
// latency-bound loop where an allocation (and the implicit synchronisation
// cudaFree brings) is not acceptable, or a process running close to a hard
// memory cap.  For them this entry point runs the same kernels as bp_loopy
// on arrays the caller already owns, and keeps its own working memory -- the
// two send buffers, the per-block delta partials and the control block -- in
// one fixed array compiled into this library.
namespace bpx {

constexpr size_t kNoAllocScratchBytes = BP_NOALLOC_SCRATCH_BYTES;

// Device-side working memory of bp_loopy_noalloc.  Every GPU that loads the
// library holds these bytes until the process exits.  In host code the name
// is only a stand-in for the symbol: the device address comes from
// cudaGetSymbolAddress on the current device, on every call, below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// device address of the scratch array on the current device.  Looked up on
// every call (a host-side table lookup): a cached address would dangle after
// a device reset reloads the module.
static int noalloc_base(void **base) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress", __FILE__, __LINE__);
    *base = p;
    return BP_OK;
}

// The caller's destination-sorted layout is checked before any kernel reads
// through it: in_ptr[0] == 0, rows non-decreasing, in_ptr[V] == E (bit 0 of
// *bad), every source id < V (bit 1).
__global__ void k_noalloc_validate(const uint32_t *__restrict__ in_ptr, const uint32_t *__restrict__ in_src,
                                   uint32_t V, uint32_t E, uint32_t *__restrict__ bad) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= V) {
        const uint32_t p = in_ptr[i];
        bool ok = i == 0 ? p == 0u : p >= in_ptr[i - 1];
        if (i == V) ok = ok && p == E;
        if (!ok) atomicOr(bad, 1u);
    }
    if (i < E && in_src[i] >= V) atomicOr(bad, 2u);
}

// scratch layout: [LoopyCtl][validation flag][partials][Q0][Q1], 256-byte
// aligned pieces
template <int MS>
static size_t noalloc_need(uint32_t V, size_t *off_bad, size_t *off_part, size_t *off_q0, size_t *qbytes) {
    constexpr int NT = flood_nt<MS>();
    *off_bad = align256(sizeof(LoopyCtl));
    *off_part = *off_bad + 256;
    *off_q0 = *off_part + align256(sizeof(double) * grid_for(V, NT));
    *qbytes = align256(sizeof(float) * MS * (size_t)V);
    return *off_q0 + 2 * *qbytes;
}

template <int MS>
static int noalloc_run(uint32_t V, uint32_t E, const uint32_t *in_ptr, const uint32_t *in_src, const float *joint,
                       float *beliefs, float *messages, int latest, int init, float tol, uint32_t max_it,
                       cudaStream_t stream, bp_loopy_result *res, int *latest_out) {
    constexpr int NT = flood_nt<MS>();
    const uint32_t grid = grid_for(V, NT);
    size_t off_bad, off_part, off_q0, qbytes;
    const size_t need = noalloc_need<MS>(V, &off_bad, &off_part, &off_q0, &qbytes);
    if (max_it > 0 && need > kNoAllocScratchBytes)
        return set_error(BP_ERR_SHAPE,
                         "bp_loopy_noalloc: %u nodes x %d states need %zu bytes of working memory; its fixed "
                         "array holds %zu (BP_NOALLOC_SCRATCH_BYTES)",
                         V, MS, need, kNoAllocScratchBytes);
    void *base = nullptr;
    int st = noalloc_base(&base);
    if (st) return st;
    unsigned char *b = (unsigned char *)base;
    LoopyCtl *ctl = (LoopyCtl *)b;
    uint32_t *bad = (uint32_t *)(b + off_bad);

    // the caller's arrays are validated first: a bad row pointer or source
    // id would otherwise be read through on the device
    BP_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), stream));
    k_noalloc_validate<<<grid_for(std::max<uint64_t>((uint64_t)V + 1, E), 256), 256, 0, stream>>>(in_ptr, in_src, V,
                                                                                                 E, bad);
    BP_CUDA(cudaGetLastError());
    uint32_t hbad = 0;
    BP_CUDA(cudaMemcpyAsync(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost, stream));
    BP_CUDA(cudaStreamSynchronize(stream));
    if (hbad & 1u)
        return set_error(BP_ERR_INVALID, "bp_loopy_noalloc: in_ptr is not a row-pointer array of %u rows ending at "
                                         "num_edges (%u)", V, E);
    if (hbad & 2u) return set_error(BP_ERR_INVALID, "bp_loopy_noalloc: a source id in in_src is >= num_nodes (%u)", V);

    float *msg_latest = messages + (size_t)latest * E * MS;
    if (init && E) {
        k_send_from_beliefs<MS, true><<<grid_for(E, 256), 256, 0, stream>>>(E, in_src, nullptr, joint, beliefs,
                                                                            msg_latest);
        BP_CUDA(cudaGetLastError());
    }
    if (max_it == 0) {
        // the reference's loop body never runs (init_previous_edge above
        // still does)
        BP_CUDA(cudaStreamSynchronize(stream));
        if (res) {
            bp_loopy_result r = {};
            r.previous_delta = -1.0f;
            *res = r;
        }
        if (latest_out) *latest_out = latest;
        return BP_OK;
    }

    // every run starts from a fully written control block; the delta
    // partials and send buffers are written before they are read
    LoopyCtl c = {};
    c.max_it = max_it;
    c.check_every = 1;
    c.msg_parity0 = (uint32_t)latest;
    c.q_parity0 = 0;
    c.serial = 0;
    c.tol = tol;
    c.prev_f = -1.0f;
    c.prev_d = -1.0;
    BP_CUDA(cudaMemcpyAsync(ctl, &c, sizeof(c), cudaMemcpyHostToDevice, stream));

    FloodArgs a = {};
    a.V = V;
    a.in_ptr = in_ptr;
    a.in_src = in_src;
    a.joint = joint;
    a.belief = beliefs;
    a.msg0 = messages;
    a.msg1 = messages + (size_t)E * MS;
    a.q0 = (float *)(b + off_q0);
    a.q1 = (float *)(b + off_q0 + qbytes);
    a.partials = (double *)(b + off_part);
    a.ctl = ctl;
    k_gather_q<MS, true><<<grid_for(V, 256), 256, 0, stream>>>(V, in_ptr, nullptr, beliefs, msg_latest, a.q0);
    BP_CUDA(cudaGetLastError());
    uint32_t done = 0;
    for (uint32_t launched = 0; launched < max_it && !done; launched += 32) {
        const uint32_t n = std::min<uint32_t>(32, max_it - launched);
        for (uint32_t i = 0; i < n; ++i) k_flood<MS, true, flood_unroll<MS>()><<<grid, NT, 0, stream>>>(a, grid);
        BP_CUDA(cudaGetLastError());
        BP_CUDA(cudaMemcpyAsync(&done, &ctl->done, sizeof(done), cudaMemcpyDeviceToHost, stream));
        BP_CUDA(cudaStreamSynchronize(stream));
    }
    BP_CUDA(cudaMemcpyAsync(&c, ctl, sizeof(c), cudaMemcpyDeviceToHost, stream));
    BP_CUDA(cudaStreamSynchronize(stream));
    if (!c.done) return set_error(BP_ERR_STATE, "loop ended without a stop decision (it=%u)", c.it);
    if (res) {
        bp_loopy_result r = {};
        r.iterations = c.ret;
        r.executed = c.it;
        r.converged = c.done == 1;
        r.delta = (float)c.delta_d;
        r.previous_delta = (float)c.prev_d;
        r.delta_f64 = c.delta_d;
        r.elapsed_ms = 0.0f;
        *res = r;
    }
    if (latest_out) *latest_out = (int)((c.msg_parity0 + c.it) & 1u);
    return BP_OK;
}

}  // namespace bpx

extern "C" int bp_loopy_noalloc(uint32_t num_nodes, uint32_t num_edges, uint32_t num_states,
                                const uint32_t *in_ptr, const uint32_t *in_src, const float *joint,
                                float *beliefs, float *messages, int latest_slot, int init_messages,
                                float tolerance, uint32_t max_iterations, void *stream, bp_loopy_result *result,
                                int *latest_out) {
    using namespace bpx;
    if (num_states < 1 || num_states > BP_MAX_STATES)
        return set_error(BP_ERR_SHAPE, "num_states %u not in [1, %d]", num_states, BP_MAX_STATES);
    if (num_nodes == 0) return set_error(BP_ERR_SHAPE, "bp_loopy_noalloc needs at least one node");
    if (!in_ptr || !beliefs || (num_edges && (!in_src || !joint || !messages)))
        return set_error(BP_ERR_INVALID, "null array");
    if (latest_slot != 0 && latest_slot != 1) return set_error(BP_ERR_INVALID, "latest_slot must be 0 or 1");
    // the kernels read S (and S*S) floats at a time as float2/float4
    if (((uintptr_t)joint | (uintptr_t)beliefs | (uintptr_t)messages) & 15u)
        return set_error(BP_ERR_INVALID, "joint, beliefs and messages must be 16-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    switch (num_states) {
    case 1: return noalloc_run<1>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    case 2: return noalloc_run<2>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    case 3: return noalloc_run<3>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    case 4: return noalloc_run<4>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    case 5: return noalloc_run<5>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    case 6: return noalloc_run<6>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    case 7: return noalloc_run<7>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    case 8: return noalloc_run<8>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    case 9: return noalloc_run<9>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    default: return noalloc_run<10>(num_nodes, num_edges, in_ptr, in_src, joint, beliefs, messages, latest_slot, init_messages, tolerance, max_iterations, s, result, latest_out);
    }
}
