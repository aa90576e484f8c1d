// unrolled.cu -- T-step unrolled loopy BP and its adjoint, in the log domain.
//
// The forward pass is the reference's update (graph.c:725-751, :1121-1183)
// on a pairwise model whose priors are softmax(log_unary) and whose joint
// tables are exp(log_pair) shared by many edges (edge e uses table
// tab[e] & 0x7f, transposed when tab[e] & 0x80), carried in logs so that
// beliefs compounding towards 0 (the reference's update multiplies the
// belief into itself every iteration) never underflow:
//   lb_0 = log_softmax(theta)
//   lm(e)[i] = r_i - LSE_i r,  r_i = LSE_j (logJ_e[i][j] + x_src[j])
//   lQ_1 = lb_0 + sum_in lm_0            (messages from x = lb_0)
//   t = 1..T:  lP = sum_in lm_t          (messages from x = lQ_t)
//              lb_t = lb_{t-1} + lP - LSE(lb_{t-1} + lP)
//              lQ_{t+1} = lb_t + lP
// The output is lb_T (log-beliefs).  The state between iterations is
// (lb, lQ); messages are recomputed from lQ wherever needed and never stored.
// The forward keeps the state every `checkpoint_every` iterations; the
// backward recomputes one segment from its checkpoint and runs the adjoint
// of each step in reverse:
//   g = lbbar_t + lQbar_{t+1};  abar = g - b_t * sum(g)  (b_t = exp lb_t)
//   lbbar_{t-1} = abar;  lPbar = abar + lQbar_{t+1};  lmbar_e = lPbar (every in-edge)
//   rbar = lmbar - m * sum(lmbar)  (m = exp lm);   w_ij = exp(logJ_ij + x_j - r_i)
//   xbar_src[j] += sum_i rbar_i w_ij;   logJbar_ij += rbar_i w_ij
// and finally theta_bar = lbbar_0 - softmax(theta) * sum(lbbar_0).
// With e_j = exp(x_j - mx) and s_i = sum_j J_ij e_j (J = exp logJ), the max
// cancels: lm_i = log s_i - log sum_k s_k, m_i = s_i / sum_k s_k and
// w_ij = J_ij e_j / s_i, so an edge costs S exponentials in either pass.
// The destination's in-edge loop, which holds e and s of the edge's
// source, writes the edge's x_src adjoint term c_j = sum_i rbar_i w_ij into
// the edge's slot of the source-sorted order; the source then sums its
// contiguous slots.  No atomics, and the result is deterministic.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bp_device.cuh"
#include "bp_internal.h"

namespace bpx {

constexpr int kUThreads = 256;
constexpr uint32_t kUMaxTables = 16;
// the adjoint kernel keeps S*S table-adjoint accumulators per thread: in
// registers for S <= 4, else in a shared-memory slice per thread (entry-major,
// so a warp's adds hit 32 different banks) with smaller blocks
template <int S> constexpr int bwd_threads() { return S <= 4 ? 256 : 64; }
// nodes per thread of the adjoint kernel (grid-stride)
constexpr uint32_t kBwdNodesPerThread = 2;
// resident blocks per SM the adjoint kernel's register allocation must allow
template <int S> constexpr int bwd_min_blocks() { return S <= 4 ? 4 : (S <= 8 ? 8 : 4); }

struct UGraph {
    uint32_t V, K;
    const uint32_t *in_ptr, *in_src, *out_ptr;
    const uint32_t *pos_out;   // slot in the source-sorted order of the edge at position p
    const uint8_t *pos_tab;
    const float *tables;   // [K][S][S] = log_pair (log joint tables)
};

// in-edges whose loads one thread issues together
template <int S> constexpr int u_batch() { return S <= 4 ? 4 : 2; }

template <int S>
__device__ __forceinline__ void load_tables_smem(const UGraph &g, float *sm) {
    // sm[2k] = exp(table k), sm[2k+1] = its transpose
    for (uint32_t i = threadIdx.x; i < g.K * S * S; i += blockDim.x) {
        const uint32_t k = i / (S * S), r = (i % (S * S)) / S, c = i % S;
        const float v = expf(g.tables[i]);
        sm[(2 * k) * S * S + r * S + c] = v;
        sm[(2 * k + 1) * S * S + c * S + r] = v;
    }
    __syncthreads();
}

template <int S>
__device__ __forceinline__ const float *edge_table(const float *sm, uint8_t tab) {
    return sm + (2u * (tab & 0x7fu) + ((tab & 0x80u) ? 1u : 0u)) * S * S;
}

template <int N>
__device__ __forceinline__ float lse(const float *a) {
    float mx = a[0];
#pragma unroll
    for (int i = 1; i < N; ++i) mx = fmaxf(mx, a[i]);
    if (mx == -INFINITY) return -INFINITY;
    float s = 0.0f;
#pragma unroll
    for (int i = 0; i < N; ++i) s += expf(a[i] - mx);
    return mx + logf(s);
}

// shifted exponentials of a log-state: e_j = exp(x_j - mx)
// (FAST: the hardware exponential __expf, a few ulp from expf; the adjoint
// uses it, the forward keeps expf)
template <int S, bool FAST = false>
__device__ __forceinline__ float shifted_exp(const float *x, float *e) {
    float mx = x[0];
#pragma unroll
    for (int j = 1; j < S; ++j) mx = fmaxf(mx, x[j]);
#pragma unroll
    for (int j = 0; j < S; ++j) e[j] = FAST ? __expf(x[j] - mx) : expf(x[j] - mx);
    return mx;
}

// row sums s_i = sum_j J_ij e_j (J linear, > 0), so r_i = mx + log s_i
template <int S>
__device__ __forceinline__ void row_sums(const float *J, const float *e, float *sr) {
#pragma unroll
    for (int i = 0; i < S; ++i) {
        float t = 0.0f;
#pragma unroll
        for (int j = 0; j < S; ++j) t += J[i * S + j] * e[j];
        sr[i] = fmaxf(t, 1e-37f);
    }
}

// message of one edge in linear form: e = exp(x - max x), row sums s of
// J e (s_i > 0); returns sum_i s_i.  lm_i = log s_i - log sum, m_i = s_i / sum.
template <int S, bool FAST = false>
__device__ __forceinline__ float msg_sums(const float *J, const float *x, float *e, float *sr) {
    shifted_exp<S, FAST>(x, e);
    row_sums<S>(J, e, sr);
    float z = 0.0f;
#pragma unroll
    for (int i = 0; i < S; ++i) z += sr[i];
    return z;
}

// P += lm over the in-edges [r0, r1) of a node, messages from the log-states
// `send`; loads of a batch of edges are issued before the first use
template <int S>
__device__ __forceinline__ void sum_log_msgs(const UGraph &g, const float *sm, const float *__restrict__ send,
                                             uint32_t r0, uint32_t r1, float *P) {
    constexpr int B = u_batch<S>();
    for (uint32_t p0 = r0; p0 < r1; p0 += B) {
        uint32_t src[B];
        uint8_t tb[B];
        float x[B][S];
#pragma unroll
        for (int b = 0; b < B; ++b)
            if (p0 + b < r1) {
                src[b] = g.in_src[p0 + b];
                tb[b] = g.pos_tab[p0 + b];
            }
#pragma unroll
        for (int b = 0; b < B; ++b)
            if (p0 + b < r1) ldv<S>(send + (size_t)src[b] * S, x[b]);
#pragma unroll
        for (int b = 0; b < B; ++b) {
            if (p0 + b >= r1) break;
            float e[S], sr[S];
            float z;
            if constexpr (S <= 4) {
                float jr[S * S];   // the edge's table, vector loads from shared memory
                ldv<S * S>(edge_table<S>(sm, tb[b]), jr);
                z = logf(msg_sums<S>(jr, x[b], e, sr));
            } else {
                z = logf(msg_sums<S>(edge_table<S>(sm, tb[b]), x[b], e, sr));
            }
#pragma unroll
            for (int i = 0; i < S; ++i) P[i] += logf(sr[i]) - z;
        }
    }
}

// sum of the x adjoint terms in the source-sorted slots [q0, q1), added in
// slot order; the loads of up to two slots are issued together
template <int S>
__device__ __forceinline__ void sum_slots(const float *__restrict__ xc, uint32_t q0, uint32_t q1, float *acc) {
    uint32_t q = q0;
    for (; q + 2 <= q1; q += 2) {
        float c0[S], c1[S];
        ldv<S>(xc + (size_t)q * S, c0);
        ldv<S>(xc + (size_t)(q + 1) * S, c1);
#pragma unroll
        for (int j = 0; j < S; ++j) acc[j] += c0[j];
#pragma unroll
        for (int j = 0; j < S; ++j) acc[j] += c1[j];
    }
    if (q < q1) {
        float c[S];
        ldv<S>(xc + (size_t)q * S, c);
#pragma unroll
        for (int j = 0; j < S; ++j) acc[j] += c[j];
    }
}

template <int S>
__global__ void k_u_logsoftmax(uint32_t V, const float *__restrict__ theta, float *__restrict__ lb0) {
    griddep_launch_dependents();
    griddep_wait();
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    float t[S];
    ldv<S>(theta + (size_t)v * S, t);
    const float z = lse<S>(t);
#pragma unroll
    for (int i = 0; i < S; ++i) t[i] -= z;
    stv<S>(lb0 + (size_t)v * S, t);
}

// lQ = lb + sum_in lm(send)   (graph.c:860-882 after :725-751)
template <int S>
__global__ void __launch_bounds__(kUThreads) k_u_gather_q(const UGraph g, const float *__restrict__ lb,
                                                          const float *__restrict__ send, float *__restrict__ lq) {
    __shared__ __align__(16) float sm[2 * kUMaxTables * S * S];
    griddep_launch_dependents();
    load_tables_smem<S>(g, sm);   // the tables do not change inside a pass
    griddep_wait();               // the kernel ahead's states
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= g.V) return;
    float qo[S];
    ldv<S>(lb + (size_t)v * S, qo);
    sum_log_msgs<S>(g, sm, send, g.in_ptr[v], g.in_ptr[v + 1], qo);
    stv<S>(lq + (size_t)v * S, qo);
}

// one forward iteration: (lb_{t-1}, lQ_t) -> (lb_t, lQ_{t+1})
template <int S>
__global__ void __launch_bounds__(kUThreads) k_u_iter(const UGraph g, const float *__restrict__ lb_in,
                                                      const float *__restrict__ lq_in, float *__restrict__ lb_out,
                                                      float *__restrict__ lq_out) {
    __shared__ __align__(16) float sm[2 * kUMaxTables * S * S];
    griddep_launch_dependents();
    load_tables_smem<S>(g, sm);
    griddep_wait();
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < g.V; v += gridDim.x * blockDim.x) {
        float P[S], a[S];
#pragma unroll
        for (int i = 0; i < S; ++i) P[i] = 0.0f;
        sum_log_msgs<S>(g, sm, lq_in, g.in_ptr[v], g.in_ptr[v + 1], P);
        ldv<S>(lb_in + (size_t)v * S, a);
#pragma unroll
        for (int i = 0; i < S; ++i) a[i] += P[i];
        const float z = lse<S>(a);
        float qo[S];
#pragma unroll
        for (int i = 0; i < S; ++i) {
            a[i] -= z;
            qo[i] = a[i] + P[i];
        }
        stv<S>(lb_out + (size_t)v * S, a);
        stv<S>(lq_out + (size_t)v * S, qo);
    }
}

// this block's sum of the per-thread table-adjoint accumulators (fixed
// order), added to its running partial row (S*S doubles); with `scale`, each
// entry k is multiplied by scale[k] first (the one-table adjoint accumulates
// ci (x) e and takes the table's factor J once per block)
template <int S, int NT, bool REG>
__device__ __forceinline__ void block_partial_add(const float *acc, const float *sacc, float (*wred)[REG ? S * S : 1],
                                                  double *__restrict__ row, const float *scale = nullptr) {
    if constexpr (REG) {
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < S * S; ++k) {
            float x = acc[k];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) wred[w][k] = x;
        }
        __syncthreads();
        for (int k = threadIdx.x; k < S * S; k += blockDim.x) {
            double t = 0.0;
            for (int ww = 0; ww < NT / 32; ++ww) t += (double)wred[ww][k];
            row[k] += scale ? (double)scale[k] * t : t;
        }
    } else {
        __syncthreads();
        for (int k = threadIdx.x; k < S * S; k += blockDim.x) {
            double t = 0.0;
            for (int tt = 0; tt < NT; ++tt) t += (double)sacc[k * NT + tt];
            row[k] += scale ? (double)scale[k] * t : t;
        }
    }
}

// the one-table form: += ci_i e_j at (i, j), or at (j, i) for a transposed
// table; the factor J at that entry is the same for every edge and is
// applied per block (block_partial_add's scale)
template <int S, int NT, bool REG>
__device__ __forceinline__ void add_table_outer(float *acc, float *sacc, const float *ci, const float *e, bool tr) {
    if constexpr (REG) {
        if (tr) {
#pragma unroll
            for (int i = 0; i < S; ++i)
#pragma unroll
                for (int j = 0; j < S; ++j) acc[j * S + i] += ci[i] * e[j];
        } else {
#pragma unroll
            for (int i = 0; i < S; ++i)
#pragma unroll
                for (int j = 0; j < S; ++j) acc[i * S + j] += ci[i] * e[j];
        }
    } else {
        const int si = tr ? 1 : S, sj = tr ? S : 1;
#pragma unroll
        for (int i = 0; i < S; ++i)
#pragma unroll
            for (int j = 0; j < S; ++j) sacc[(i * si + j * sj) * NT + threadIdx.x] += ci[i] * e[j];
    }
}

// table adjoint of the edge with scaled adjoint ci (rbar_i / s_i), table J
// and source exponentials e: += ci_i J_ij e_j at (i, j), or at (j, i) for a
// transposed table
template <int S, int NT, bool REG>
__device__ __forceinline__ void add_table_adjoint(float *acc, float *sacc, const float *ci, const float *J,
                                                  const float *e, bool tr) {
    if constexpr (REG) {
        if (tr) {
#pragma unroll
            for (int i = 0; i < S; ++i)
#pragma unroll
                for (int j = 0; j < S; ++j) acc[j * S + i] += ci[i] * J[i * S + j] * e[j];
        } else {
#pragma unroll
            for (int i = 0; i < S; ++i)
#pragma unroll
                for (int j = 0; j < S; ++j) acc[i * S + j] += ci[i] * J[i * S + j] * e[j];
        }
    } else {
        const int si = tr ? 1 : S, sj = tr ? S : 1;
#pragma unroll
        for (int i = 0; i < S; ++i)
#pragma unroll
            for (int j = 0; j < S; ++j) sacc[(i * si + j * sj) * NT + threadIdx.x] += ci[i] * J[i * S + j] * e[j];
    }
}

// several tables (K > 1): table k's adjoint, from the per-node Pbar the
// adjoint kernel stored; every in-edge with table k recomputes its message
// sums.  One launch per table keeps the accumulators per thread.
template <int S>
__global__ void __launch_bounds__(bwd_threads<S>()) k_u_pair_grad(const UGraph g, const float *__restrict__ send,
                                                                  const float *__restrict__ pbar, uint32_t k,
                                                                  double *__restrict__ epart_k) {
    constexpr int NT = bwd_threads<S>();
    constexpr bool REG = S <= 4;
    __shared__ __align__(16) float sm[2 * kUMaxTables * S * S];
    __shared__ float sacc[REG ? 1 : S * S * NT];
    __shared__ float wred[NT / 32][REG ? S * S : 1];
    griddep_launch_dependents();
    load_tables_smem<S>(g, sm);
    griddep_wait();
    float acc[REG ? S * S : 1];
    if constexpr (REG) {
#pragma unroll
        for (int q = 0; q < S * S; ++q) acc[q] = 0.0f;
    } else {
        for (int q = 0; q < S * S; ++q) sacc[q * NT + threadIdx.x] = 0.0f;
    }
    for (uint32_t v = blockIdx.x * NT + threadIdx.x; v < g.V; v += gridDim.x * NT) {
        float Pb[S], ps = 0.0f;
        ldv<S>(pbar + (size_t)v * S, Pb);
#pragma unroll
        for (int i = 0; i < S; ++i) ps += Pb[i];
        for (uint32_t p = g.in_ptr[v]; p < g.in_ptr[v + 1]; ++p) {
            const uint8_t tab = g.pos_tab[p];
            if ((tab & 0x7fu) != k) continue;
            float x[S], e[S], sr[S], ci[S];
            ldv<S>(send + (size_t)g.in_src[p] * S, x);
            const float *J = edge_table<S>(sm, tab);
            const float z = msg_sums<S, true>(J, x, e, sr);
            const float psz = __fdividef(ps, z);
#pragma unroll
            for (int i = 0; i < S; ++i) ci[i] = __fdividef(Pb[i], sr[i]) - psz;
            add_table_adjoint<S, NT, REG>(acc, sacc, ci, J, e, (tab & 0x80u) != 0);
        }
    }
    block_partial_add<S, NT, REG>(acc, sacc, wred, epart_k + (size_t)blockIdx.x * S * S);
}

// node step of the adjoint at node v: lbbar_{t-1}(v) (to lbbar_out) and
// Pbar = the adjoint of the node's summed log-messages, from lbbar_t(v) and
// lQbar_{t+1}(v) (the gather of iteration t+1's x adjoint terms in v's
// source-sorted slots); mode 1 is the initial step lQ_1 = lb_0 + lP
template <int S>
__device__ __forceinline__ void bwd_node_step(const UGraph &g, int mode, uint32_t v, const float *__restrict__ lb_t,
                                              const float *__restrict__ lbbar_t, const float *__restrict__ xc_next,
                                              float *__restrict__ lbbar_out, float *__restrict__ pbar_out,
                                              float *Pbar) {
    float gb[S], gq[S];
#pragma unroll
    for (int i = 0; i < S; ++i) {
        gb[i] = 0.0f;
        gq[i] = 0.0f;
    }
    if (lbbar_t) ldv<S>(lbbar_t + (size_t)v * S, gb);
    if (xc_next) sum_slots<S>(xc_next, g.out_ptr[v], g.out_ptr[v + 1], gq);
    float out[S];
    if (mode == 0) {
        float lb[S], gs = 0.0f;
        ldv<S>(lb_t + (size_t)v * S, lb);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            gb[i] += gq[i];
            gs += gb[i];
        }
#pragma unroll
        for (int i = 0; i < S; ++i) {
            out[i] = gb[i] - expf(lb[i]) * gs;
            Pbar[i] = out[i] + gq[i];
        }
    } else {
#pragma unroll
        for (int i = 0; i < S; ++i) {
            out[i] = gb[i] + gq[i];
            Pbar[i] = gq[i];
        }
    }
    stv<S>(lbbar_out + (size_t)v * S, out);
    if (pbar_out) stv<S>(pbar_out + (size_t)v * S, Pbar);   // several tables: k_u_pair_grad's input
}

// one in-edge's adjoint quantities: e (source exponentials), ci = rbar_i / s_i
// and the x adjoint terms c_j = e_j sum_i ci_i J_ij, for table J (the edge's,
// transposed when the edge says so) and log-state x of the source
template <int S>
__device__ __forceinline__ void bwd_edge(const float *J, const float *x, const float *Pbar, float ps, float *e,
                                         float *ci, float *c) {
    float sr[S];
    const float z = msg_sums<S, true>(J, x, e, sr);
    // rbar_i / s_i = (Pbar_i - (s_i / z) sum(Pbar)) / s_i = Pbar_i / s_i - sum(Pbar) / z
    // (fast division: s_i and z lie in [1e-37, S max J])
    const float psz = __fdividef(ps, z);
#pragma unroll
    for (int i = 0; i < S; ++i) ci[i] = __fdividef(Pbar[i], sr[i]) - psz;
#pragma unroll
    for (int j = 0; j < S; ++j) c[j] = 0.0f;
#pragma unroll
    for (int i = 0; i < S; ++i)
#pragma unroll
        for (int j = 0; j < S; ++j) c[j] += ci[i] * J[i * S + j];
#pragma unroll
    for (int j = 0; j < S; ++j) c[j] *= e[j];
}

// adjoint of iteration t at node v (mode 0), or of the initial step
// (mode 1: lQ_1 = lb_0 + lP, messages from send = lb_0), fused with the
// gather of lQbar_{t+1}(v) from iteration t+1's x adjoint terms (xc_next, in
// source-sorted slots; null at t = T).  Writes lbbar_out (mode 1: lbbar_0
// without its own send term), this iteration's x adjoint terms xc, and adds
// the block's log-table adjoint into epart.
template <int S, int B = 2, int MB = bwd_min_blocks<S>()>
__global__ void __launch_bounds__(bwd_threads<S>(), MB) k_u_bwd(const UGraph g, int mode, const float *__restrict__ send,
                                                           const float *__restrict__ lb_t,
                                                           const float *__restrict__ lbbar_t,
                                                           const float *__restrict__ xc_next,
                                                           float *__restrict__ lbbar_out, float *__restrict__ xc,
                                                           double *__restrict__ epart, float *__restrict__ pbar_out) {
    constexpr int NT = bwd_threads<S>();
    constexpr bool REG = S <= 4;
    __shared__ __align__(16) float sm[2 * kUMaxTables * S * S];
    __shared__ float sacc[REG ? 1 : S * S * NT];
    __shared__ float wred[NT / 32][REG ? S * S : 1];
    griddep_launch_dependents();
    load_tables_smem<S>(g, sm);
    griddep_wait();
    float acc[REG ? S * S : 1];
    if constexpr (REG) {
#pragma unroll
        for (int k = 0; k < S * S; ++k) acc[k] = 0.0f;
    } else {
        for (int k = 0; k < S * S; ++k) sacc[k * NT + threadIdx.x] = 0.0f;
    }
    // grid-stride over nodes: several nodes per thread share one block
    // reduction of the table adjoint
    for (uint32_t v = blockIdx.x * NT + threadIdx.x; v < g.V; v += gridDim.x * NT) {
        // the in-edge range first: its loads overlap the node step's
        const uint32_t r0 = g.in_ptr[v], r1 = g.in_ptr[v + 1];
        float Pbar[S];
        bwd_node_step<S>(g, mode, v, lb_t, lbbar_t, xc_next, lbbar_out, pbar_out, Pbar);
        const bool one_table = pbar_out == nullptr;
        float ps = 0.0f;
#pragma unroll
        for (int i = 0; i < S; ++i) ps += Pbar[i];
        for (uint32_t p0 = r0; p0 < r1; p0 += B) {
            uint32_t src[B], slot[B];
            uint8_t tb[B];
            float x[B][S];
#pragma unroll
            for (int b = 0; b < B; ++b)
                if (p0 + b < r1) {
                    src[b] = g.in_src[p0 + b];
                    tb[b] = g.pos_tab[p0 + b];
                    slot[b] = g.pos_out[p0 + b];
                }
#pragma unroll
            for (int b = 0; b < B; ++b)
                if (p0 + b < r1) ldv<S>(send + (size_t)src[b] * S, x[b]);
#pragma unroll
            for (int b = 0; b < B; ++b) {
                if (p0 + b >= r1) break;
                const float *Js = edge_table<S>(sm, tb[b]);
                float jr[S <= 4 ? S * S : 1];
                if constexpr (S <= 4) ldv<S * S>(Js, jr);   // the edge's table in registers
                const float *J = S <= 4 ? jr : Js;
                float e[S], ci[S], c[S];
                bwd_edge<S>(J, x[b], Pbar, ps, e, ci, c);
                if (one_table) add_table_outer<S, NT, REG>(acc, sacc, ci, e, (tb[b] & 0x80u) != 0);
                stv<S>(xc + (size_t)slot[b] * S, c);
            }
        }
    }
    // several tables: k_u_pair_grad adds the table adjoint
    if (pbar_out) return;
    block_partial_add<S, NT, REG>(acc, sacc, wred, epart + (size_t)blockIdx.x * S * S, sm);
}

// ---- the one-table adjoint on the tensor cores (5 <= S <= 8) ------------
// With one shared table J, the table adjoint is J (.) sum over edges of
// ci (x) e (transposed edges into the transposed entry), i.e. C^T E for the
// edges' ci and e rows: a GEMM with K = the number of edges.  Each warp stages
// 32 edges (one per lane) per round in shared memory and accumulates
// D (16 x 8) += A (16 x 32) B (32 x 8) with four mma.sync m16n8k8 TF32 steps;
// rows 0-7 of A hold ci of the non-transposed edges, rows 8-15 ci of the
// transposed ones, B holds e (both zero-padded to 8 states).  Each product
// is split into TF32 high and low parts (3 MMAs: hi*hi + hi*lo + lo*hi), which
// keeps it to about fp32 accuracy; accumulation is fp32.  The order of every
// sum is fixed, so the result is deterministic.
constexpr int kMmaThreads = 128;

__device__ __forceinline__ uint32_t to_tf32(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ void split_tf32(float x, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32(x);
    lo = to_tf32(x - __uint_as_float(hi));
}

__device__ __forceinline__ void mma_tf32_16x8x8(float *d, const uint32_t *a, const uint32_t *b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// PF 1: the in-edge range and the first in-edge's source state are loaded
// ahead of the node step, and each round loads the next round's in-edge
// (table id, slot, source state) before it works on its own, so the gather
// of the source state overlaps a round of arithmetic
template <int S, int PF = 1>
__global__ void __launch_bounds__(kMmaThreads, 4) k_u_bwd_mma(const UGraph g, int mode, const float *__restrict__ send,
                                                             const float *__restrict__ lb_t,
                                                             const float *__restrict__ lbbar_t,
                                                             const float *__restrict__ xc_next,
                                                             float *__restrict__ lbbar_out, float *__restrict__ xc,
                                                             double *__restrict__ epart) {
    static_assert(S >= 1 && S <= 8, "states padded to 8");
    constexpr int NW = kMmaThreads / 32;
    __shared__ __align__(16) float sm[2 * kUMaxTables * S * S];
    __shared__ __align__(16) float st_c[NW][32][8];
    __shared__ __align__(16) float st_e[NW][32][8];
    __shared__ float st_tr[NW][32];
    __shared__ float dred[NW][16][8];
    griddep_launch_dependents();
    load_tables_smem<S>(g, sm);
    griddep_wait();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gq = lane >> 2, tq = lane & 3;
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (uint32_t base = (blockIdx.x * NW + warp) * 32u;; base += gridDim.x * (uint32_t)kMmaThreads) {
        const uint32_t v = base + lane;
        const bool active = v < g.V;
        if (!__any_sync(0xffffffffu, active)) break;
        float Pbar[S], ps = 0.0f;
        uint32_t r0 = 0, r1 = 0;
        uint8_t ntab = 0;   // PF: the next in-edge's table id, slot and source state
        uint32_t nslot = 0;
        float nx[S];
        if (active) {
            if constexpr (PF) {
                r0 = g.in_ptr[v];
                r1 = g.in_ptr[v + 1];
                if (r0 < r1) {
                    ntab = g.pos_tab[r0];
                    nslot = g.pos_out[r0];
                    ldv<S>(send + (size_t)g.in_src[r0] * S, nx);
                }
            }
            bwd_node_step<S>(g, mode, v, lb_t, lbbar_t, xc_next, lbbar_out, nullptr, Pbar);
#pragma unroll
            for (int i = 0; i < S; ++i) ps += Pbar[i];
            if constexpr (!PF) {
                r0 = g.in_ptr[v];
                r1 = g.in_ptr[v + 1];
            }
        }
        for (uint32_t j = 0;; ++j) {
            const bool has = r0 + j < r1;
            if (!__any_sync(0xffffffffu, has)) break;
            float cs[8], es[8], tr = 0.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                cs[i] = 0.0f;
                es[i] = 0.0f;
            }
            if (has) {
                const uint32_t p = r0 + j;
                uint8_t tab;
                uint32_t slot;
                float x[S], e[S], ci[S], c[S];
                if constexpr (PF) {
                    tab = ntab;
                    slot = nslot;
#pragma unroll
                    for (int i = 0; i < S; ++i) x[i] = nx[i];
                    if (p + 1 < r1) {
                        ntab = g.pos_tab[p + 1];
                        nslot = g.pos_out[p + 1];
                        ldv<S>(send + (size_t)g.in_src[p + 1] * S, nx);
                    }
                } else {
                    tab = g.pos_tab[p];
                    slot = g.pos_out[p];
                    ldv<S>(send + (size_t)g.in_src[p] * S, x);
                }
                bwd_edge<S>(edge_table<S>(sm, tab), x, Pbar, ps, e, ci, c);
                stv<S>(xc + (size_t)slot * S, c);
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    cs[i] = ci[i];
                    es[i] = e[i];
                }
                tr = (tab & 0x80u) ? 1.0f : 0.0f;
            }
            reinterpret_cast<float4 *>(st_c[warp][lane])[0] = make_float4(cs[0], cs[1], cs[2], cs[3]);
            reinterpret_cast<float4 *>(st_c[warp][lane])[1] = make_float4(cs[4], cs[5], cs[6], cs[7]);
            reinterpret_cast<float4 *>(st_e[warp][lane])[0] = make_float4(es[0], es[1], es[2], es[3]);
            reinterpret_cast<float4 *>(st_e[warp][lane])[1] = make_float4(es[4], es[5], es[6], es[7]);
            st_tr[warp][lane] = tr;
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                // A (16 x 8, row-major): a0 (g, t), a1 (g+8, t), a2 (g, t+4), a3 (g+8, t+4)
                // B (8 x 8, column-major): b0 (t, g), b1 (t+4, g); k indexes the round's edges
                const int k0 = q * 8 + tq, k1 = k0 + 4;
                const float c0 = st_c[warp][k0][gq], c1 = st_c[warp][k1][gq];
                const bool t0 = st_tr[warp][k0] != 0.0f, t1 = st_tr[warp][k1] != 0.0f;
                const float af[4] = {t0 ? 0.0f : c0, t0 ? c0 : 0.0f, t1 ? 0.0f : c1, t1 ? c1 : 0.0f};
                const float bf[2] = {st_e[warp][k0][gq], st_e[warp][k1][gq]};
                uint32_t ah[4], al[4], bh[2], bl[2];
#pragma unroll
                for (int i = 0; i < 4; ++i) split_tf32(af[i], ah[i], al[i]);
#pragma unroll
                for (int i = 0; i < 2; ++i) split_tf32(bf[i], bh[i], bl[i]);
                mma_tf32_16x8x8(d, ah, bh);
                mma_tf32_16x8x8(d, ah, bl);
                mma_tf32_16x8x8(d, al, bh);
            }
            __syncwarp();
        }
    }
    // D (16 x 8): d0 (g, 2t), d1 (g, 2t+1), d2 (g+8, 2t), d3 (g+8, 2t+1)
    dred[warp][gq][2 * tq] = d[0];
    dred[warp][gq][2 * tq + 1] = d[1];
    dred[warp][gq + 8][2 * tq] = d[2];
    dred[warp][gq + 8][2 * tq + 1] = d[3];
    __syncthreads();
    // logJbar[a][b] += J[a][b] * (N[a][b] + T[b][a]), J = exp(table 0)
    for (int k = threadIdx.x; k < S * S; k += blockDim.x) {
        const int ra = k / S, cb = k % S;
        double t = 0.0;
        for (int w = 0; w < NW; ++w) t += (double)dred[w][ra][cb] + (double)dred[w][8 + cb][ra];
        epart[(size_t)blockIdx.x * S * S + k] += (double)sm[ra * S + cb] * t;
    }
}

// ---- the one-table adjoint in pull form (one table, S <= 8) --------------
// With one table J an edge's message depends only on its source's state and
// the table's orientation (J or J^T), so a source can gather the x adjoint
// of its out-edges itself instead of each destination scattering a per-edge
// term into a slot.  For source u with e = exp(x_u - max), the row sums
// sN = J e and sT = J^T e and their totals zN, zT (once per node, not once
// per in-edge), and each out-edge u -> w of orientation o:
//   ci = Pbar(w) / s_o - sum(Pbar(w)) / z_o
// summed over the out-edges into cN (J edges) and cT (J^T edges):
//   xbar_u[j] = e_j * sum_i (cN_i J_ij + cT_i J_ji)
//   logJbar  += J (.) (cN (x) e + (cT (x) e)^T)
// The kernel of step t finishes step t+1's edges from Pbar_{t+1} of the
// out-neighbours (the previous launch's output) and then runs step t's node
// step, writing Pbar_t: no E x S slot arrays, and the per-edge DRAM traffic
// is the out-neighbour's id, the table id and the (cached) Pbar gather.
//   mode 0, step t:  g = lbbar_t + xbar;  lbbar_{t-1} = g - b_t sum(g);
//                    Pbar_t = lbbar_{t-1} + xbar            (x = lQ_{t+1})
//   mode 1, lQ_1 = lb_0 + lP:  lbbar_0 = gin + xbar;  Pbar = xbar   (x = lQ_1)
//   mode 2, priors:  a = gin + xbar;  theta_bar = a - softmax(theta) sum(a),
//                    softmax(theta) = exp(lb_0)                  (x = lb_0)
// x_next null (t = T): no out-edge terms.  Tables: S <= 4 keeps the S*S
// accumulators in registers; 5 <= S <= 8 sums cN (x) e and cT (x) e of 32
// nodes per warp round on the tensor cores as k_u_bwd_mma does.
constexpr int kPullThreads = 128;
// resident blocks per SM the pull kernel's registers are capped for.  5-8
// states, 256 grids of 8 states: 25.1 ms forward+backward at 4, 24.0 at 5,
// 25.0 at 6 (spills).  4 states, the 512x512 grid: 0.847 ms at 4 (86
// registers), 0.837 at 6, 0.785 at 8 (64 registers, 44 B of spills)
template <int S> constexpr int pull_min_blocks() { return S <= 4 ? 8 : 5; }

template <int S>
__device__ __forceinline__ void pull_out_edges(const UGraph &g, const uint32_t *__restrict__ out_dst,
                                               const uint8_t *__restrict__ out_tab, const float *sm,
                                               const float *__restrict__ pbar_next, uint32_t u, const float *x,
                                               float *e, float *cn, float *ct, float *xbar) {
    const uint32_t q0 = g.out_ptr[u], q1 = g.out_ptr[u + 1];
    shifted_exp<S, true>(x, e);
    float rn[S], rt[S], zn = 0.0f, zt = 0.0f;
    row_sums<S>(sm, e, rn);
    row_sums<S>(sm + S * S, e, rt);
#pragma unroll
    for (int i = 0; i < S; ++i) {
        zn += rn[i];
        zt += rt[i];
    }
    // reciprocals once per node (s_i and z lie in [1e-37, S max J])
#pragma unroll
    for (int i = 0; i < S; ++i) {
        rn[i] = __fdividef(1.0f, rn[i]);
        rt[i] = __fdividef(1.0f, rt[i]);
        cn[i] = 0.0f;
        ct[i] = 0.0f;
    }
    const float izn = __fdividef(1.0f, zn), izt = __fdividef(1.0f, zt);
    for (uint32_t q = q0; q < q1; q += 2) {
        const bool two = q + 1 < q1;
        const uint32_t w0 = out_dst[q], w1 = two ? out_dst[q + 1] : w0;
        const bool t0 = (out_tab[q] & 0x80u) != 0, t1 = two && (out_tab[q + 1] & 0x80u) != 0;
        float p0[S], p1[S];
        ldv<S>(pbar_next + (size_t)w0 * S, p0);
        ldv<S>(pbar_next + (size_t)w1 * S, p1);
        float s0 = 0.0f, s1 = 0.0f;
#pragma unroll
        for (int i = 0; i < S; ++i) {
            s0 += p0[i];
            s1 += p1[i];
        }
        const float a0 = s0 * (t0 ? izt : izn), a1 = s1 * (t1 ? izt : izn);
#pragma unroll
        for (int i = 0; i < S; ++i) {
            const float c = p0[i] * (t0 ? rt[i] : rn[i]) - a0;
            cn[i] += t0 ? 0.0f : c;
            ct[i] += t0 ? c : 0.0f;
        }
        if (two) {
#pragma unroll
            for (int i = 0; i < S; ++i) {
                const float c = p1[i] * (t1 ? rt[i] : rn[i]) - a1;
                cn[i] += t1 ? 0.0f : c;
                ct[i] += t1 ? c : 0.0f;
            }
        }
    }
    // the tables are read again from shared memory here rather than kept in
    // registers across the out-edge loop (2 S^2 values)
    asm volatile("" ::: "memory");
#pragma unroll
    for (int j = 0; j < S; ++j) {
        float t = 0.0f;
#pragma unroll
        for (int i = 0; i < S; ++i) t += cn[i] * sm[i * S + j] + ct[i] * sm[S * S + i * S + j];
        xbar[j] = e[j] * t;
    }
}

template <int S, int MB = pull_min_blocks<S>()>
__global__ void __launch_bounds__(kPullThreads, MB) k_u_bwd_pull(
    const UGraph g, const uint32_t *__restrict__ out_dst, const uint8_t *__restrict__ out_tab, int mode,
    const float *__restrict__ x_next, const float *__restrict__ pbar_next, const float *__restrict__ lb_t,
    const float *__restrict__ gin, float *__restrict__ gout, float *__restrict__ pbar_out, double *__restrict__ epart) {
    static_assert(S >= 1 && S <= 8, "pull form: up to 8 states");
    constexpr bool MMA = S >= 5;
    constexpr int NT = kPullThreads, NW = NT / 32;
    __shared__ __align__(16) float sm[2 * S * S];   // J and J^T
    __shared__ __align__(16) float st_n[MMA ? NW : 1][32][8];
    __shared__ __align__(16) float st_t[MMA ? NW : 1][32][8];
    __shared__ __align__(16) float st_e[MMA ? NW : 1][32][8];
    __shared__ float dred[MMA ? NW : 1][16][8];
    __shared__ float wred[NW][MMA ? 1 : S * S];
    griddep_launch_dependents();
    load_tables_smem<S>(g, sm);
    griddep_wait();
    const bool edges = x_next != nullptr;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, gq = lane >> 2, tq = lane & 3;
    float acc[MMA ? 1 : S * S];
#pragma unroll
    for (int k = 0; k < (MMA ? 1 : S * S); ++k) acc[k] = 0.0f;
    float d[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    for (uint32_t base = (blockIdx.x * NW + warp) * 32u;; base += gridDim.x * (uint32_t)NT) {
        const uint32_t u = base + lane;
        const bool active = u < g.V;
        if (!__any_sync(0xffffffffu, active)) break;
        float e[S], cn[S], ct[S], xb[S];
#pragma unroll
        for (int i = 0; i < S; ++i) {
            e[i] = 0.0f;
            cn[i] = 0.0f;
            ct[i] = 0.0f;
            xb[i] = 0.0f;
        }
        if (active) {
            float gi[S], lb[S];
            ldv<S>(gin + (size_t)u * S, gi);
            if (mode == 0) ldv<S>(lb_t + (size_t)u * S, lb);
            if (edges) {
                float x[S];
                ldv<S>(x_next + (size_t)u * S, x);
                pull_out_edges<S>(g, out_dst, out_tab, sm, pbar_next, u, x, e, cn, ct, xb);
            }
            if (mode == 2) ldv<S>(x_next + (size_t)u * S, lb);   // lb_0 (an L1 hit)
            float out[S], pb[S], gs = 0.0f;
#pragma unroll
            for (int i = 0; i < S; ++i) {
                gi[i] += xb[i];
                gs += gi[i];
            }
            if (mode == 0) {
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    out[i] = gi[i] - expf(lb[i]) * gs;
                    pb[i] = out[i] + xb[i];
                }
            } else if (mode == 1) {
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    out[i] = gi[i];
                    pb[i] = xb[i];
                }
            } else {
#pragma unroll
                for (int i = 0; i < S; ++i) out[i] = gi[i] - expf(lb[i]) * gs;
            }
            stv<S>(gout + (size_t)u * S, out);
            if (mode != 2) stv<S>(pbar_out + (size_t)u * S, pb);
            if constexpr (!MMA) {
                if (edges) {
#pragma unroll
                    for (int i = 0; i < S; ++i)
#pragma unroll
                        for (int j = 0; j < S; ++j) acc[i * S + j] += cn[i] * e[j] + ct[j] * e[i];
                }
            }
        }
        if constexpr (MMA) {
            if (edges) {
                // A (16 x 32 nodes): rows 0-7 cN, rows 8-15 cT; B (32 nodes x 8): e
                float pn[8], pt[8], pe[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    pn[i] = 0.0f;
                    pt[i] = 0.0f;
                    pe[i] = 0.0f;
                }
#pragma unroll
                for (int i = 0; i < S; ++i) {
                    pn[i] = cn[i];
                    pt[i] = ct[i];
                    pe[i] = e[i];
                }
                reinterpret_cast<float4 *>(st_n[warp][lane])[0] = make_float4(pn[0], pn[1], pn[2], pn[3]);
                reinterpret_cast<float4 *>(st_n[warp][lane])[1] = make_float4(pn[4], pn[5], pn[6], pn[7]);
                reinterpret_cast<float4 *>(st_t[warp][lane])[0] = make_float4(pt[0], pt[1], pt[2], pt[3]);
                reinterpret_cast<float4 *>(st_t[warp][lane])[1] = make_float4(pt[4], pt[5], pt[6], pt[7]);
                reinterpret_cast<float4 *>(st_e[warp][lane])[0] = make_float4(pe[0], pe[1], pe[2], pe[3]);
                reinterpret_cast<float4 *>(st_e[warp][lane])[1] = make_float4(pe[4], pe[5], pe[6], pe[7]);
                __syncwarp();
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int k0 = q * 8 + tq, k1 = k0 + 4;
                    const float af[4] = {st_n[warp][k0][gq], st_t[warp][k0][gq], st_n[warp][k1][gq],
                                         st_t[warp][k1][gq]};
                    const float bf[2] = {st_e[warp][k0][gq], st_e[warp][k1][gq]};
                    uint32_t ah[4], al[4], bh[2], bl[2];
#pragma unroll
                    for (int i = 0; i < 4; ++i) split_tf32(af[i], ah[i], al[i]);
#pragma unroll
                    for (int i = 0; i < 2; ++i) split_tf32(bf[i], bh[i], bl[i]);
                    mma_tf32_16x8x8(d, ah, bh);
                    mma_tf32_16x8x8(d, ah, bl);
                    mma_tf32_16x8x8(d, al, bh);
                }
                __syncwarp();
            }
        }
    }
    if (!edges) return;   // uniform over the grid: no table adjoint in this launch
    if constexpr (MMA) {
        dred[warp][gq][2 * tq] = d[0];
        dred[warp][gq][2 * tq + 1] = d[1];
        dred[warp][gq + 8][2 * tq] = d[2];
        dred[warp][gq + 8][2 * tq + 1] = d[3];
        __syncthreads();
        // logJbar[a][b] += J[a][b] * (N[a][b] + T[b][a])
        for (int k = threadIdx.x; k < S * S; k += NT) {
            const int ra = k / S, cb = k % S;
            double t = 0.0;
            for (int w = 0; w < NW; ++w) t += (double)dred[w][ra][cb] + (double)dred[w][8 + cb][ra];
            epart[(size_t)blockIdx.x * S * S + k] += (double)sm[ra * S + cb] * t;
        }
    } else {
        block_partial_add<S, NT, true>(acc, nullptr, wred, epart + (size_t)blockIdx.x * S * S, sm);
    }
}

// the initial step's end: lbbar_0(s) = add(s) + the x adjoint terms of s's
// out-edges, then through the log-softmax of the priors:
// theta_bar = lbbar_0 - softmax(theta) * sum(lbbar_0)
template <int S>
__global__ void __launch_bounds__(kUThreads) k_u_bwd_src(const UGraph g, const float *__restrict__ xc,
                                                         const float *__restrict__ add, const float *__restrict__ lb0,
                                                         float *__restrict__ theta_bar) {
    griddep_launch_dependents();
    griddep_wait();
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.V) return;
    float acc[S], lb[S], sum = 0.0f;
    ldv<S>(add + (size_t)s * S, acc);
    sum_slots<S>(xc, g.out_ptr[s], g.out_ptr[s + 1], acc);
    ldv<S>(lb0 + (size_t)s * S, lb);
#pragma unroll
    for (int i = 0; i < S; ++i) sum += acc[i];
#pragma unroll
    for (int i = 0; i < S; ++i) acc[i] = acc[i] - expf(lb[i]) * sum;
    stv<S>(theta_bar + (size_t)s * S, acc);
}

// log_pair_bar[k] = sum of the block partials (fixed order): one block per
// entry; partials laid out [table][block][S*S]
__global__ void k_u_reduce_pair(const double *__restrict__ epart, uint32_t nblk, uint32_t ss, float *__restrict__ out) {
    __shared__ double red[32];
    griddep_launch_dependents();
    griddep_wait();
    const uint32_t k = blockIdx.x, kt = k / ss, idx = k % ss;
    const double *base = epart + (size_t)kt * nblk * ss + idx;
    double t = 0.0;
    for (uint32_t b = threadIdx.x; b < nblk; b += blockDim.x) t += base[(size_t)b * ss];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) s += red[w];
        out[k] = (float)s;
    }
}

}  // namespace bpx

struct bp_unrolled {
    uint32_t V = 0, E = 0, S = 0, K = 0, T = 0, ck = 1, nck = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t *in_ptr = nullptr, *in_src = nullptr, *out_ptr = nullptr, *pos_out = nullptr;
    uint8_t *pos_tab = nullptr;
    float *tables = nullptr;
    float *ck_b = nullptr, *ck_q = nullptr;    // [nck][V][S]
    float *seg_b = nullptr, *seg_q = nullptr;  // [2][ck][V][S] (slot 0 unused), by segment parity
    cudaStream_t side = nullptr;                // the backward's recompute stream
    cudaEvent_t ev_fork = nullptr, ev_rec[2] = {nullptr, nullptr}, ev_bwd[2] = {nullptr, nullptr};
    float *pp_b = nullptr, *pp_q = nullptr;    // [2][V][S]
    float *bT = nullptr;
    float *bbar[2] = {nullptr, nullptr};
    float *xc[2] = {nullptr, nullptr};       // [E][S] x adjoint terms, source-sorted slots (scatter form)
    bool pull = false;                       // the adjoint in pull form (one table, S <= 8)
    uint32_t *out_dst = nullptr;             // [E] destination of source-sorted slot q (pull form)
    uint8_t *out_tab = nullptr;              // [E] its table id (pull form)
    float *pbv[2] = {nullptr, nullptr};      // [V][S] Pbar of steps t and t+1 (pull form)
    float *pbar = nullptr;                   // [V][S] node-step adjoint Pbar (several tables only)
    double *epart = nullptr;
    float *theta_buf = nullptr, *gtheta_buf = nullptr, *glogp_buf = nullptr;
    cudaGraphExec_t fwd_exec = nullptr, bwd_exec = nullptr;
    uint32_t nblk = 0;
    bool forward_done = false;
    float fwd_ms = 0.0f, bwd_ms = 0.0f;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace bpx {

// Launches of the forward and backward passes use programmatic dependent
// launch: each kernel lets the next one start once all its blocks run; the
// next kernel loads and exponentiates the tables (which no kernel of a pass
// writes) and then waits (griddepcontrol.wait) for the whole grid ahead and
// its memory before it reads any state.  BP_UNROLLED_PDL=0 turns it off.
static bool u_pdl() {
    static int on = -1;
    if (on < 0) {
        const char *env = getenv("BP_UNROLLED_PDL");
        on = (env && env[0] == '0') ? 0 : 1;
    }
    return on != 0;
}

template <typename... KArgs, typename... Args>
static int u_launch(void (*kern)(KArgs...), unsigned grid, unsigned block, cudaStream_t st, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = u_pdl() ? 1 : 0;
    cudaError_t e = cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...);
    if (e != cudaSuccess) return cuda_fail(e, "cudaLaunchKernelEx", __FILE__, __LINE__);
    return BP_OK;
}

// in-edges per batch of the adjoint kernel (BP_UBWD_BATCH=2|4, 1-4 states)
// and nodes per thread (BP_UBWD_NPT=1|2); every choice gives the same results
static int ubwd_env(const char *name, int dflt, int alt) {
    const char *env = getenv(name);
    return (env && atoi(env) == alt) ? alt : dflt;
}

// the forward on the engine's own buffers (theta_buf, tables): captured once
// into a CUDA graph, replayed on every call
template <int S>
static int u_forward(bp_unrolled *u) {
    const UGraph g{u->V, u->K, u->in_ptr, u->in_src, u->out_ptr, u->pos_out, u->pos_tab, u->tables};
    const size_t VS = (size_t)u->V * S;
    const unsigned gv = grid_for(u->V, kUThreads);
    cudaStream_t st = u->stream;
    int rc;
    if ((rc = u_launch(k_u_logsoftmax<S>, gv, kUThreads, st, u->V, (const float *)u->theta_buf, u->ck_b))) return rc;
    if ((rc = u_launch(k_u_gather_q<S>, gv, kUThreads, st, g, (const float *)u->ck_b, (const float *)u->ck_b,
                       u->ck_q)))
        return rc;
    // state t (lb_t, lQ_{t+1}) lives in checkpoint slot t/ck when t % ck == 0;
    // inside the last segment in its slot of the segment buffer, where the
    // backward reads it without recomputing; else in pp[t&1]
    const uint32_t nseg = (u->T + u->ck - 1) / u->ck, t0_last = (nseg - 1) * u->ck;
    const size_t last_buf = (size_t)((nseg - 1) & 1u) * u->ck;
    auto loc_b = [&](uint32_t t) {
        if (t % u->ck == 0) return u->ck_b + (t / u->ck) * VS;
        if (t > t0_last) return u->seg_b + (last_buf + (t - t0_last)) * VS;
        return u->pp_b + (t & 1) * VS;
    };
    auto loc_q = [&](uint32_t t) {
        if (t % u->ck == 0) return u->ck_q + (t / u->ck) * VS;
        if (t > t0_last) return u->seg_q + (last_buf + (t - t0_last)) * VS;
        return u->pp_q + (t & 1) * VS;
    };
    for (uint32_t t = 1; t <= u->T; ++t) {
        float *bo = (t == u->T) ? u->bT : loc_b(t);
        float *qo = (t == u->T) ? u->pp_q + (t & 1) * VS : loc_q(t);
        if ((rc = u_launch(k_u_iter<S>, gv, kUThreads, st, g, (const float *)loc_b(t - 1), (const float *)loc_q(t - 1),
                           bo, qo)))
            return rc;
    }
    return BP_OK;
}

// the backward on the engine's own buffers (bbar[0] holds d loss / d lb_T on
// entry; gtheta_buf, glogp_buf receive the gradients)
// the backward in pull form (one table, S <= 8; see k_u_bwd_pull): kernel t
// finishes step t+1's edges and runs step t's node step; then the initial
// gather (mode 1) and the priors (mode 2).  Recompute and segment buffers as
// in the scatter form below.
template <int S>
static int u_backward_pull(bp_unrolled *u) {
    if constexpr (S > 8) {
        return set_error(BP_ERR_STATE, "pull form with %d states", S);
    } else {
        const UGraph g{u->V, u->K, u->in_ptr, u->in_src, u->out_ptr, u->pos_out, u->pos_tab, u->tables};
        const size_t VS = (size_t)u->V * S;
        const unsigned gv = grid_for(u->V, kUThreads);
        const unsigned gp = grid_for(u->V, kPullThreads * 2);
        cudaStream_t st = u->stream;
        int rc = BP_OK;
        BP_CUDA(cudaMemsetAsync(u->epart, 0, sizeof(double) * gp * S * S, st));
        // 4-8 states: the register cap, in resident blocks per SM, may be set
        // to 4, 5, 6 or 8 (BP_UBWD_PULL_MB; default pull_min_blocks)
        int mb = 0;
        if (S >= 4) {
            const char *env = getenv("BP_UBWD_PULL_MB");
            mb = env ? atoi(env) : 0;
        }
        auto step = [&](int mode, const float *xn, const float *pn, const float *b_t, const float *gin, float *gout,
                        float *pout) -> int {
            const uint32_t *od = u->out_dst;
            const uint8_t *ot = u->out_tab;
            if constexpr (S >= 4) {
                switch (mb) {
                case 4: return u_launch(k_u_bwd_pull<S, 4>, gp, kPullThreads, st, g, od, ot, mode, xn, pn, b_t, gin,
                                        gout, pout, u->epart);
                case 5: return u_launch(k_u_bwd_pull<S, 5>, gp, kPullThreads, st, g, od, ot, mode, xn, pn, b_t, gin,
                                        gout, pout, u->epart);
                case 6: return u_launch(k_u_bwd_pull<S, 6>, gp, kPullThreads, st, g, od, ot, mode, xn, pn, b_t, gin,
                                        gout, pout, u->epart);
                case 8: return u_launch(k_u_bwd_pull<S, 8>, gp, kPullThreads, st, g, od, ot, mode, xn, pn, b_t, gin,
                                        gout, pout, u->epart);
                default: break;
                }
            }
            return u_launch(k_u_bwd_pull<S>, gp, kPullThreads, st, g, od, ot, mode, xn, pn, b_t, gin, gout, pout,
                            u->epart);
        };
        const uint32_t nseg = (u->T + u->ck - 1) / u->ck;
        auto seg_b = [&](uint32_t s, uint32_t j) { return u->seg_b + ((size_t)(s & 1u) * u->ck + j) * VS; };
        auto seg_q = [&](uint32_t s, uint32_t j) { return u->seg_q + ((size_t)(s & 1u) * u->ck + j) * VS; };
        auto recompute = [&](uint32_t s) -> int {
            const uint32_t t0 = s * u->ck, t_end = std::min(t0 + u->ck, u->T);
            const float *ckb = u->ck_b + (size_t)s * VS, *ckq = u->ck_q + (size_t)s * VS;
            for (uint32_t j = 1; j + t0 < t_end; ++j) {
                const float *bi = (j == 1) ? ckb : seg_b(s, j - 1);
                const float *qi = (j == 1) ? ckq : seg_q(s, j - 1);
                int r = u_launch(k_u_iter<S>, gv, kUThreads, u->side, g, bi, qi, seg_b(s, j), seg_q(s, j));
                if (r) return r;
            }
            return BP_OK;
        };
        int bc = 0, pc = 0;
        const float *pn = nullptr;   // Pbar of step t+1 (none at t = T)
        BP_CUDA(cudaEventRecord(u->ev_fork, st));
        BP_CUDA(cudaStreamWaitEvent(u->side, u->ev_fork, 0));
        BP_CUDA(cudaEventRecord(u->ev_rec[(nseg - 1) & 1u], u->side));
        for (int s = (int)nseg - 1; s >= 0; --s) {
            if (s >= 1) {
                if ((uint32_t)s + 1 < nseg) BP_CUDA(cudaStreamWaitEvent(u->side, u->ev_bwd[(s + 1) & 1], 0));
                if ((rc = recompute((uint32_t)s - 1))) return rc;
                BP_CUDA(cudaEventRecord(u->ev_rec[(s - 1) & 1], u->side));
            }
            BP_CUDA(cudaStreamWaitEvent(st, u->ev_rec[s & 1], 0));
            const uint32_t t0 = (uint32_t)s * u->ck, t_end = std::min(t0 + u->ck, u->T);
            for (uint32_t t = t_end; t > t0; --t) {
                const uint32_t j = t - t0 - 1;
                const float *b_t = (t == u->T) ? u->bT
                                   : (t == t_end) ? u->ck_b + (size_t)(s + 1) * VS
                                                  : seg_b((uint32_t)s, j + 1);   // lb_t
                // lQ_{t+1}: the next segment's checkpoint after the segment's last step
                const float *q_next = (t == u->T) ? nullptr
                                      : (t == t_end) ? u->ck_q + (size_t)(s + 1) * VS
                                                     : seg_q((uint32_t)s, j + 1);
                if ((rc = step(0, q_next, pn, b_t, u->bbar[bc], u->bbar[bc ^ 1], u->pbv[pc]))) return rc;
                bc ^= 1;
                pn = u->pbv[pc];
                pc ^= 1;
            }
            BP_CUDA(cudaEventRecord(u->ev_bwd[s & 1], st));
        }
        BP_CUDA(cudaGetLastError());
        // step 1's edges (x = lQ_1, checkpoint 0) and the initial gather lQ_1 = lb_0 + lP
        if ((rc = step(1, u->ck_q, pn, nullptr, u->bbar[bc], u->bbar[bc ^ 1], u->pbv[pc]))) return rc;
        bc ^= 1;
        pn = u->pbv[pc];
        // the initial gather's edges (x = lb_0) and the priors' log-softmax
        if ((rc = step(2, u->ck_b, pn, nullptr, u->bbar[bc], u->gtheta_buf, nullptr))) return rc;
        return u_launch(k_u_reduce_pair, S * S, 256u, st, (const double *)u->epart, gp, (uint32_t)(S * S),
                        u->glogp_buf);
    }
}

template <int S>
static int u_backward(bp_unrolled *u) {
    const UGraph g{u->V, u->K, u->in_ptr, u->in_src, u->out_ptr, u->pos_out, u->pos_tab, u->tables};
    const size_t VS = (size_t)u->V * S;
    const unsigned gv = grid_for(u->V, kUThreads);
    constexpr int BT = bwd_threads<S>();
    // one table and 5..8 states: the table adjoint on the tensor cores
    const bool mma = S >= 5 && S <= 8 && u->K == 1;
    // the tensor-core adjoint's in-edge loads one round ahead (BP_UBWD_PF=0: in the round that uses them)
    const bool mma_pf = ubwd_env("BP_UBWD_PF", 1, 0) == 1;
    const int batch = S <= 4 ? ubwd_env("BP_UBWD_BATCH", 2, 4) : 2;
    const uint32_t npt = (uint32_t)ubwd_env("BP_UBWD_NPT", (int)kBwdNodesPerThread, 1);
    // register cap of the adjoint kernel, 1-4 states: BP_UBWD_MINB=3 allows
    // 85 registers (3 blocks per SM) instead of 64 (4 blocks)
    const int minb = ubwd_env("BP_UBWD_MINB", 4, 3);
    const unsigned gb = mma ? grid_for(u->V, kMmaThreads * 2) : grid_for(u->V, BT * npt);
    // the recompute keeps the forward's grid, a thread per node: on smaller
    // grids beside the adjoint (80-296 blocks) it became the critical path
    const unsigned rgrid = gv;
    cudaStream_t st = u->stream;
    int rc = BP_OK;
    auto adjoint = [&](int mode, const float *send, const float *b_t, const float *gbar, const float *xn, float *out,
                       float *xo, float *pb) -> int {
        if constexpr (S >= 5 && S <= 8) {
            if (mma && mma_pf)
                return u_launch(k_u_bwd_mma<S, 1>, gb, kMmaThreads, st, g, mode, send, b_t, gbar, xn, out, xo,
                                u->epart);
            if (mma) return u_launch(k_u_bwd_mma<S, 0>, gb, kMmaThreads, st, g, mode, send, b_t, gbar, xn, out, xo,
                                     u->epart);
        }
        if constexpr (S <= 4) {
            if (batch == 4)
                return u_launch(k_u_bwd<S, 4>, gb, BT, st, g, mode, send, b_t, gbar, xn, out, xo, u->epart, pb);
            if (minb == 3)
                return u_launch(k_u_bwd<S, 2, 3>, gb, BT, st, g, mode, send, b_t, gbar, xn, out, xo, u->epart, pb);
        }
        return u_launch(k_u_bwd<S, 2>, gb, BT, st, g, mode, send, b_t, gbar, xn, out, xo, u->epart, pb);
    };
    if (u->pull) return u_backward_pull<S>(u);
    BP_CUDA(cudaMemsetAsync(u->epart, 0, sizeof(double) * u->K * gb * S * S, st));
    // several tables: the table adjoint of each backward step, one pass per table
    auto pair_grads = [&](const float *send) -> int {
        for (uint32_t k = 0; u->K > 1 && k < u->K; ++k) {
            int r = u_launch(k_u_pair_grad<S>, gb, BT, st, g, send, (const float *)u->pbar, k,
                             u->epart + (size_t)k * gb * S * S);
            if (r) return r;
        }
        return BP_OK;
    };
    float *pbar = u->K > 1 ? u->pbar : nullptr;
    int bc = 0, rn = 0;
    const float *xc_next = nullptr;   // x adjoint terms of iteration t+1 (none at t = T)
    const uint32_t nseg = (u->T + u->ck - 1) / u->ck;
    // Segment s's recompute needs only its checkpoint, so it runs on the side
    // stream while the adjoint of segment s+1 runs on the main stream; the
    // two share nothing but the double-buffered segment states (buffer s & 1)
    auto seg_b = [&](uint32_t s, uint32_t j) { return u->seg_b + ((size_t)(s & 1u) * u->ck + j) * VS; };
    auto seg_q = [&](uint32_t s, uint32_t j) { return u->seg_q + ((size_t)(s & 1u) * u->ck + j) * VS; };
    auto recompute = [&](uint32_t s) -> int {
        const uint32_t t0 = s * u->ck, t_end = std::min(t0 + u->ck, u->T);
        const float *ckb = u->ck_b + (size_t)s * VS, *ckq = u->ck_q + (size_t)s * VS;
        for (uint32_t j = 1; j + t0 < t_end; ++j) {
            const float *bi = (j == 1) ? ckb : seg_b(s, j - 1);
            const float *qi = (j == 1) ? ckq : seg_q(s, j - 1);
            int r = u_launch(k_u_iter<S>, rgrid, kUThreads, u->side, g, bi, qi, seg_b(s, j), seg_q(s, j));
            if (r) return r;
        }
        return BP_OK;
    };
    // the last segment's states are the forward's own (u_forward)
    BP_CUDA(cudaEventRecord(u->ev_fork, st));
    BP_CUDA(cudaStreamWaitEvent(u->side, u->ev_fork, 0));
    BP_CUDA(cudaEventRecord(u->ev_rec[(nseg - 1) & 1u], u->side));
    for (int s = (int)nseg - 1; s >= 0; --s) {
        if (s >= 1) {
            // buffer (s-1)&1 was last read by the adjoint of segment s+1
            if ((uint32_t)s + 1 < nseg) BP_CUDA(cudaStreamWaitEvent(u->side, u->ev_bwd[(s + 1) & 1], 0));
            if ((rc = recompute((uint32_t)s - 1))) return rc;
            BP_CUDA(cudaEventRecord(u->ev_rec[(s - 1) & 1], u->side));
        }
        BP_CUDA(cudaStreamWaitEvent(st, u->ev_rec[s & 1], 0));
        const uint32_t t0 = (uint32_t)s * u->ck, t_end = std::min(t0 + u->ck, u->T);
        const float *ckq = u->ck_q + (size_t)s * VS;
        for (uint32_t t = t_end; t > t0; --t) {
            const uint32_t j = t - t0 - 1;
            const float *q_t = (j == 0) ? ckq : seg_q((uint32_t)s, j);       // lQ_t
            const float *b_t = (t == u->T) ? u->bT
                               : (t == t_end) ? u->ck_b + (size_t)(s + 1) * VS
                                              : seg_b((uint32_t)s, j + 1);  // lb_t
            if ((rc = adjoint(0, q_t, b_t, u->bbar[bc], xc_next, u->bbar[bc ^ 1], u->xc[rn], pbar))) return rc;
            if ((rc = pair_grads(q_t))) return rc;
            bc ^= 1;
            xc_next = u->xc[rn];
            rn ^= 1;
        }
        BP_CUDA(cudaEventRecord(u->ev_bwd[s & 1], st));
    }
    BP_CUDA(cudaGetLastError());
    // initial step: lQ_1 = lb_0 + sum lm(lb_0); its own x adjoint goes to lb_0
    const float *b0 = u->ck_b;
    if ((rc = adjoint(1, b0, nullptr, u->bbar[bc], xc_next, u->bbar[bc ^ 1], u->xc[rn], pbar))) return rc;
    if ((rc = pair_grads(b0))) return rc;
    if ((rc = u_launch(k_u_bwd_src<S>, gv, kUThreads, st, g, (const float *)u->xc[rn], (const float *)u->bbar[bc ^ 1],
                       b0, u->gtheta_buf)))
        return rc;
    return u_launch(k_u_reduce_pair, u->K * S * S, 256u, st, (const double *)u->epart, gb, (uint32_t)(S * S),
                    u->glogp_buf);
}

static void u_free(bp_unrolled *u) {
    if (!u) return;
    void *ptrs[] = {u->in_ptr, u->in_src, u->out_ptr, u->pos_out, u->pos_tab, u->tables, u->ck_b, u->ck_q,
                    u->seg_b, u->seg_q, u->pp_b, u->pp_q, u->bT, u->bbar[0], u->bbar[1], u->xc[0],
                    u->xc[1], u->epart, u->theta_buf, u->gtheta_buf, u->glogp_buf, u->pbar, u->out_dst,
                    u->out_tab, u->pbv[0], u->pbv[1]};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (u->fwd_exec) cudaGraphExecDestroy(u->fwd_exec);
    if (u->bwd_exec) cudaGraphExecDestroy(u->bwd_exec);
    if (u->ev0) cudaEventDestroy(u->ev0);
    if (u->ev1) cudaEventDestroy(u->ev1);
    cudaEvent_t evs[] = {u->ev_fork, u->ev_rec[0], u->ev_rec[1], u->ev_bwd[0], u->ev_bwd[1]};
    for (cudaEvent_t e : evs)
        if (e) cudaEventDestroy(e);
    if (u->side) cudaStreamDestroy(u->side);
    if (u->own_stream && u->stream) cudaStreamDestroy(u->stream);
    delete u;
}

}  // namespace bpx

using namespace bpx;

#define BP_DISPATCH_S(S_, FN, ...)                                 \
    switch (S_) {                                                  \
    case 1: return FN<1>(__VA_ARGS__);                             \
    case 2: return FN<2>(__VA_ARGS__);                             \
    case 3: return FN<3>(__VA_ARGS__);                             \
    case 4: return FN<4>(__VA_ARGS__);                             \
    case 5: return FN<5>(__VA_ARGS__);                             \
    case 6: return FN<6>(__VA_ARGS__);                             \
    case 7: return FN<7>(__VA_ARGS__);                             \
    case 8: return FN<8>(__VA_ARGS__);                             \
    case 9: return FN<9>(__VA_ARGS__);                             \
    default: return FN<10>(__VA_ARGS__);                           \
    }

// ---- the cross-entropy loss head: -mean_v log_beliefs[v][label_v] -------
// one launch for the value (per-block partials in f64, the last block sums
// them in block order, so the value is deterministic) and one for its
// gradient (-g / V at each node's label, 0 elsewhere), instead of a gather,
// a reduction and a scatter of generic tensor kernels
constexpr int kNllThreads = 256;
constexpr uint32_t kNllBlocks = 296;   // 2 per SM

__global__ void __launch_bounds__(kNllThreads) k_nll(const float *__restrict__ lb, const int64_t *__restrict__ labels,
                                                      uint32_t V, uint32_t S, double *partials, uint32_t *ticket,
                                                      float *loss) {
    __shared__ double red[kNllThreads / 32];
    __shared__ bool last;
    double acc = 0.0;
    for (uint32_t v = blockIdx.x * kNllThreads + threadIdx.x; v < V; v += gridDim.x * kNllThreads) {
        const uint64_t lab = (uint64_t)labels[v];   // a label outside [0, S) makes the loss NaN
        acc -= lab < S ? (double)lb[(size_t)v * S + lab] : __longlong_as_double(0x7ff8000000000000ll);
    }
    double t = block_sum<kNllThreads>(acc, red);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = t;
        unsigned k;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(k) : "l"(ticket) : "memory");
        last = (k == gridDim.x - 1);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double a = 0.0;
    for (uint32_t k = threadIdx.x; k < gridDim.x; k += kNllThreads) a += __ldcg(partials + k);
    a = block_sum<kNllThreads>(a, red);
    if (threadIdx.x == 0) {
        *loss = (float)(a / (double)V);
        *ticket = 0;
    }
}

__global__ void k_nll_grad(const int64_t *__restrict__ labels, uint32_t V, uint32_t S, const float *__restrict__ g,
                           float *__restrict__ grad) {
    const uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= (uint64_t)V * S) return;
    const uint32_t v = (uint32_t)(k / S), st = (uint32_t)(k % S);
    grad[k] = ((uint64_t)st == (uint64_t)labels[v]) ? -g[0] / (float)V : 0.0f;
}

extern "C" {

int bp_nll_f32(const float *log_beliefs, const int64_t *labels, uint32_t V, uint32_t S, double *scratch,
               float *loss, void *stream) {
    if (!log_beliefs || !labels || !scratch || !loss) return set_error(BP_ERR_INVALID, "null argument");
    if (V == 0 || S == 0) return set_error(BP_ERR_SHAPE, "empty log-beliefs");
    // scratch: kNllBlocks partials, then the ticket (zero before the first call)
    k_nll<<<kNllBlocks, kNllThreads, 0, (cudaStream_t)stream>>>(log_beliefs, labels, V, S, scratch,
                                                               reinterpret_cast<uint32_t *>(scratch + kNllBlocks),
                                                               loss);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

int bp_nll_grad_f32(const int64_t *labels, uint32_t V, uint32_t S, const float *grad_loss, float *grad_log_beliefs,
                    void *stream) {
    if (!labels || !grad_loss || !grad_log_beliefs) return set_error(BP_ERR_INVALID, "null argument");
    const uint64_t n = (uint64_t)V * S;
    if (n) k_nll_grad<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(labels, V, S, grad_loss, grad_log_beliefs);
    BP_CUDA(cudaGetLastError());
    return BP_OK;
}

int bp_unrolled_create(bp_unrolled **out, uint32_t V, uint32_t E, uint32_t S, uint32_t K, const uint32_t *src,
                       const uint32_t *dst, const uint8_t *tab, uint32_t T, uint32_t ck, void *stream) {
    if (!out || (E && (!src || !dst || !tab))) return set_error(BP_ERR_INVALID, "null argument");
    *out = nullptr;
    if (S < 1 || S > BP_MAX_STATES) return set_error(BP_ERR_SHAPE, "num_states %u", S);
    if (K < 1 || K > kUMaxTables) return set_error(BP_ERR_SHAPE, "num_tables %u not in [1, %u]", K, kUMaxTables);
    if (V == 0 || T == 0) return set_error(BP_ERR_SHAPE, "need nodes and at least one iteration");
    if (ck == 0) ck = 1;
    for (uint32_t e = 0; e < E; ++e) {
        if (src[e] >= V || dst[e] >= V) return set_error(BP_ERR_INVALID, "edge %u endpoint out of range", e);
        if ((tab[e] & 0x7fu) >= K) return set_error(BP_ERR_INVALID, "edge %u table %u >= %u", e, tab[e] & 0x7f, K);
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_error(BP_ERR_NO_DEVICE, "no CUDA device");
    bp_unrolled *u = new bp_unrolled();
    u->V = V, u->E = E, u->S = S, u->K = K, u->T = T, u->ck = ck;
    u->nck = (T - 1) / ck + 1;
    if (stream) {
        u->stream = (cudaStream_t)stream;
    } else {
        cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking);
        u->own_stream = true;
    }
    // destination-sorted (stable) and source-sorted edge orders, on the host
    std::vector<uint32_t> in_ptr(V + 1, 0), out_ptr(V + 1, 0), in_src(E), pos_out(E);
    std::vector<uint8_t> ptab(E);
    for (uint32_t e = 0; e < E; ++e) {
        in_ptr[dst[e] + 1]++;
        out_ptr[src[e] + 1]++;
    }
    for (uint32_t v = 0; v < V; ++v) {
        in_ptr[v + 1] += in_ptr[v];
        out_ptr[v + 1] += out_ptr[v];
    }
    std::vector<uint32_t> fill(in_ptr.begin(), in_ptr.end() - 1), pos_of(E);
    for (uint32_t e = 0; e < E; ++e) {
        const uint32_t p = fill[dst[e]]++;
        pos_of[e] = p;
        in_src[p] = src[e];
        ptab[p] = tab[e];
    }
    std::vector<uint32_t> ofill(out_ptr.begin(), out_ptr.end() - 1);
    for (uint32_t e = 0; e < E; ++e) pos_out[pos_of[e]] = ofill[src[e]]++;
    // one table and up to 8 states: the adjoint in pull form (BP_UBWD_PULL=0: the scatter form)
    u->pull = K == 1 && S <= 8 && ubwd_env("BP_UBWD_PULL", 1, 0) == 1;
    std::vector<uint32_t> odst;
    std::vector<uint8_t> otab;
    if (u->pull) {
        odst.resize(E);
        otab.resize(E);
        for (uint32_t e = 0; e < E; ++e) {
            const uint32_t q = pos_out[pos_of[e]];
            odst[q] = dst[e];
            otab[q] = tab[e];
        }
    }
    const size_t VS = (size_t)V * S;
    u->nblk = grid_for(V, 64);   // partial slots for the smallest backward block
    auto alloc = [&](void **p, size_t bytes) {
        return cudaMalloc(p, bytes ? bytes : 16) == cudaSuccess;
    };
    bool ok = alloc((void **)&u->in_ptr, sizeof(uint32_t) * (V + 1)) && alloc((void **)&u->in_src, 4 * (size_t)E) &&
              alloc((void **)&u->out_ptr, sizeof(uint32_t) * (V + 1)) && alloc((void **)&u->pos_out, 4 * (size_t)E) &&
              alloc((void **)&u->pos_tab, (size_t)E) && alloc((void **)&u->tables, sizeof(float) * K * S * S) &&
              alloc((void **)&u->ck_b, sizeof(float) * VS * u->nck) &&
              alloc((void **)&u->ck_q, sizeof(float) * VS * u->nck) &&
              alloc((void **)&u->seg_b, sizeof(float) * VS * 2 * ck) &&
              alloc((void **)&u->seg_q, sizeof(float) * VS * 2 * ck) &&
              alloc((void **)&u->pp_b, sizeof(float) * VS * 2) && alloc((void **)&u->pp_q, sizeof(float) * VS * 2) &&
              alloc((void **)&u->bT, sizeof(float) * VS) && alloc((void **)&u->bbar[0], sizeof(float) * VS) &&
              alloc((void **)&u->bbar[1], sizeof(float) * VS) &&
              (u->pull || (alloc((void **)&u->xc[0], sizeof(float) * S * (size_t)E) &&
                           alloc((void **)&u->xc[1], sizeof(float) * S * (size_t)E))) &&
              (!u->pull || (alloc((void **)&u->out_dst, 4 * (size_t)E) && alloc((void **)&u->out_tab, (size_t)E) &&
                            alloc((void **)&u->pbv[0], sizeof(float) * VS) &&
                            alloc((void **)&u->pbv[1], sizeof(float) * VS))) &&
              alloc((void **)&u->epart, sizeof(double) * K * u->nblk * S * S) &&
              (K == 1 || alloc((void **)&u->pbar, sizeof(float) * VS)) &&
              alloc((void **)&u->theta_buf, sizeof(float) * VS) && alloc((void **)&u->gtheta_buf, sizeof(float) * VS) &&
              alloc((void **)&u->glogp_buf, sizeof(float) * K * S * S);
    if (!ok) {
        u_free(u);
        return set_error(BP_ERR_NOMEM, "device allocation failed for the unrolled graph");
    }
    cudaMemcpyAsync(u->in_ptr, in_ptr.data(), 4 * (V + 1), cudaMemcpyHostToDevice, u->stream);
    cudaMemcpyAsync(u->out_ptr, out_ptr.data(), 4 * (V + 1), cudaMemcpyHostToDevice, u->stream);
    if (E) {
        cudaMemcpyAsync(u->in_src, in_src.data(), 4 * (size_t)E, cudaMemcpyHostToDevice, u->stream);
        cudaMemcpyAsync(u->pos_out, pos_out.data(), 4 * (size_t)E, cudaMemcpyHostToDevice, u->stream);
        cudaMemcpyAsync(u->pos_tab, ptab.data(), (size_t)E, cudaMemcpyHostToDevice, u->stream);
        if (u->pull) {
            cudaMemcpyAsync(u->out_dst, odst.data(), 4 * (size_t)E, cudaMemcpyHostToDevice, u->stream);
            cudaMemcpyAsync(u->out_tab, otab.data(), (size_t)E, cudaMemcpyHostToDevice, u->stream);
        }
    }
    cudaEventCreate(&u->ev0);
    cudaEventCreate(&u->ev1);
    bool evok = cudaStreamCreateWithFlags(&u->side, cudaStreamNonBlocking) == cudaSuccess &&
                cudaEventCreateWithFlags(&u->ev_fork, cudaEventDisableTiming) == cudaSuccess;
    for (int i = 0; i < 2 && evok; ++i)
        evok = cudaEventCreateWithFlags(&u->ev_rec[i], cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&u->ev_bwd[i], cudaEventDisableTiming) == cudaSuccess;
    if (!evok) {
        u_free(u);
        return set_error(BP_ERR_CUDA, "stream or event creation failed");
    }
    if (cudaStreamSynchronize(u->stream) != cudaSuccess) {
        u_free(u);
        return set_error(BP_ERR_CUDA, "upload of the unrolled graph failed");
    }
    *out = u;
    return BP_OK;
}

void bp_unrolled_destroy(bp_unrolled *u) {
    if (!u) return;
    cudaStreamSynchronize(u->stream);
    u_free(u);
}

static int capture(bp_unrolled *u, cudaGraphExec_t *exec, int (*body)(bp_unrolled *)) {
    cudaGraph_t graph = nullptr;
    BP_CUDA(cudaStreamBeginCapture(u->stream, cudaStreamCaptureModeThreadLocal));
    int st = body(u);
    cudaError_t ce = cudaStreamEndCapture(u->stream, &graph);
    if (st) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (ce != cudaSuccess) return cuda_fail(ce, "cudaStreamEndCapture", __FILE__, __LINE__);
    cudaError_t ie = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) return cuda_fail(ie, "cudaGraphInstantiate", __FILE__, __LINE__);
    return BP_OK;
}

static int fwd_body(bp_unrolled *u) { BP_DISPATCH_S(u->S, u_forward, u); }
static int bwd_body(bp_unrolled *u) { BP_DISPATCH_S(u->S, u_backward, u); }

int bp_unrolled_forward(bp_unrolled *u, const float *log_unary, const float *log_pair, float *log_beliefs) {
    NvtxRange nvtx("bp_unrolled_forward");
    if (!u || !log_unary || !log_pair || !log_beliefs) return set_error(BP_ERR_INVALID, "null argument");
    if (((uintptr_t)log_unary | (uintptr_t)log_beliefs) & 15u)
        return set_error(BP_ERR_INVALID, "log_unary and log_beliefs must be 16-byte aligned");
    const size_t VS = (size_t)u->V * u->S;
    BP_CUDA(cudaMemcpyAsync(u->theta_buf, log_unary, sizeof(float) * VS, cudaMemcpyDeviceToDevice, u->stream));
    BP_CUDA(cudaMemcpyAsync(u->tables, log_pair, sizeof(float) * u->K * u->S * u->S, cudaMemcpyDeviceToDevice,
                            u->stream));
    int st;
    if (!u->fwd_exec && (st = capture(u, &u->fwd_exec, fwd_body))) return st;
    BP_CUDA(cudaGraphLaunch(u->fwd_exec, u->stream));
    BP_CUDA(cudaMemcpyAsync(log_beliefs, u->bT, sizeof(float) * VS, cudaMemcpyDeviceToDevice, u->stream));
    u->forward_done = true;
    return BP_OK;
}

int bp_unrolled_backward(bp_unrolled *u, const float *grad_log_beliefs, float *grad_log_unary, float *grad_log_pair) {
    NvtxRange nvtx("bp_unrolled_backward");
    if (!u || !grad_log_beliefs || !grad_log_unary || !grad_log_pair) return set_error(BP_ERR_INVALID, "null argument");
    if (((uintptr_t)grad_log_beliefs | (uintptr_t)grad_log_unary) & 15u)
        return set_error(BP_ERR_INVALID, "grad_log_beliefs and grad_log_unary must be 16-byte aligned");
    if (!u->forward_done) return set_error(BP_ERR_STATE, "backward before forward");
    const size_t VS = (size_t)u->V * u->S;
    BP_CUDA(cudaMemcpyAsync(u->bbar[0], grad_log_beliefs, sizeof(float) * VS, cudaMemcpyDeviceToDevice, u->stream));
    int st;
    if (!u->bwd_exec && (st = capture(u, &u->bwd_exec, bwd_body))) return st;
    BP_CUDA(cudaGraphLaunch(u->bwd_exec, u->stream));
    BP_CUDA(cudaMemcpyAsync(grad_log_unary, u->gtheta_buf, sizeof(float) * VS, cudaMemcpyDeviceToDevice, u->stream));
    BP_CUDA(cudaMemcpyAsync(grad_log_pair, u->glogp_buf, sizeof(float) * u->K * u->S * u->S,
                            cudaMemcpyDeviceToDevice, u->stream));
    return BP_OK;
}

int bp_unrolled_set_stream(bp_unrolled *u, void *stream) {
    if (!u) return set_error(BP_ERR_INVALID, "null argument");
    BP_CUDA(cudaStreamSynchronize(u->stream));
    if (u->own_stream) cudaStreamDestroy(u->stream);
    u->own_stream = false;
    if (stream) {
        u->stream = (cudaStream_t)stream;
    } else {
        BP_CUDA(cudaStreamCreateWithFlags(&u->stream, cudaStreamNonBlocking));
        u->own_stream = true;
    }
    return BP_OK;
}

}  // extern "C"
