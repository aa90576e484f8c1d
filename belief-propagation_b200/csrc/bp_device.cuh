// bp_device.cuh -- device helpers shared by the loopy, tree and build kernels.
//
// Arithmetic parity: every product, sum and quotient that the reference
// computes in fp32 is written with the round-to-nearest intrinsics
// (__fmul_rn / __fadd_rn / __fsub_rn / __fdiv_rn), which nvcc never fuses
// into FMA, in the reference's order.  Results are then bit-identical to the
// reference compiled with gcc on x86-64 (SSE, no contraction).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "bp_internal.h"

namespace bpx {

#define FMUL __fmul_rn
#define FADD __fadd_rn
#define FSUB __fsub_rn
#define FDIV __fdiv_rn

// ---- vector loads / stores of N consecutive floats ------------------------
// N*4 bytes at an address that is a multiple of N*4 bytes (every array here is
// indexed by element * N), so float4 needs N % 4 == 0 and float2 N % 2 == 0.
enum CacheHint { kDefault = 0, kStream = 1, kReadOnly = 2 };

template <int N, int H = kDefault>
__device__ __forceinline__ void ldv(const float *__restrict__ p, float *o) {
    if constexpr (N % 4 == 0) {
#pragma unroll
        for (int k = 0; k < N / 4; ++k) {
            float4 v;
            if constexpr (H == kStream) v = __ldcs(reinterpret_cast<const float4 *>(p) + k);
            else if constexpr (H == kReadOnly) v = __ldg(reinterpret_cast<const float4 *>(p) + k);
            else v = reinterpret_cast<const float4 *>(p)[k];
            o[4 * k] = v.x; o[4 * k + 1] = v.y; o[4 * k + 2] = v.z; o[4 * k + 3] = v.w;
        }
    } else if constexpr (N % 2 == 0) {
#pragma unroll
        for (int k = 0; k < N / 2; ++k) {
            float2 v;
            if constexpr (H == kStream) v = __ldcs(reinterpret_cast<const float2 *>(p) + k);
            else if constexpr (H == kReadOnly) v = __ldg(reinterpret_cast<const float2 *>(p) + k);
            else v = reinterpret_cast<const float2 *>(p)[k];
            o[2 * k] = v.x; o[2 * k + 1] = v.y;
        }
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            if constexpr (H == kStream) o[k] = __ldcs(p + k);
            else if constexpr (H == kReadOnly) o[k] = __ldg(p + k);
            else o[k] = p[k];
        }
    }
}

template <int N, int H = kDefault>
__device__ __forceinline__ void stv(float *__restrict__ p, const float *v) {
    if constexpr (N % 4 == 0) {
#pragma unroll
        for (int k = 0; k < N / 4; ++k) {
            float4 w = make_float4(v[4 * k], v[4 * k + 1], v[4 * k + 2], v[4 * k + 3]);
            if constexpr (H == kStream) __stcs(reinterpret_cast<float4 *>(p) + k, w);
            else reinterpret_cast<float4 *>(p)[k] = w;
        }
    } else if constexpr (N % 2 == 0) {
#pragma unroll
        for (int k = 0; k < N / 2; ++k) {
            float2 w = make_float2(v[2 * k], v[2 * k + 1]);
            if constexpr (H == kStream) __stcs(reinterpret_cast<float2 *>(p) + k, w);
            else reinterpret_cast<float2 *>(p)[k] = w;
        }
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            if constexpr (H == kStream) __stcs(p + k, v[k]);
            else p[k] = v[k];
        }
    }
}

// ---- the send step ---------------------------------------------------------
// m[i] = sum_j J[i][j] * buf[j] for i < x, j < y (partial sums from 0 in j
// order), normalised by their sum over i (sum <= 0 replaced by 1):
// graph.c:884-910 (send_message_for_edge), :426-448 (send_message).
// buf slots at or beyond the source's state count are zero (the reference
// reads stale slots there, graph.c:851-857).  Slots i >= x come out 0.
// the same arithmetic on a table already held in registers (row-major MS x MS)
template <int MS, bool UNI>
__device__ __forceinline__ void send_msg_regs(const float *j, const float *buf, int x, int y, float *m) {
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < MS; ++i) {
        float partial = 0.0f;
        if (UNI || i < x) {
#pragma unroll
            for (int c = 0; c < MS; ++c)
                if (UNI || c < y) partial = FADD(partial, FMUL(j[i * MS + c], buf[c]));
            sum = FADD(sum, partial);
        }
        m[i] = partial;
    }
    if (sum <= 0.0f) sum = 1.0f;
#pragma unroll
    for (int i = 0; i < MS; ++i) m[i] = (UNI || i < x) ? FDIV(m[i], sum) : 0.0f;
}

template <int MS, bool UNI>
__device__ __forceinline__ void send_msg(const float *__restrict__ J, const float *buf, int x, int y,
                                         float *m) {
    float sum = 0.0f;
    if constexpr (MS * MS <= 16) {
        float j[MS * MS];
        ldv<MS * MS, kStream>(J, j);
#pragma unroll
        for (int i = 0; i < MS; ++i) {
            float partial = 0.0f;
            if (UNI || i < x) {
#pragma unroll
                for (int c = 0; c < MS; ++c)
                    if (UNI || c < y) partial = FADD(partial, FMUL(j[i * MS + c], buf[c]));
                sum = FADD(sum, partial);
            }
            m[i] = partial;
        }
    } else {
#pragma unroll
        for (int i = 0; i < MS; ++i) {
            float partial = 0.0f;
            if (UNI || i < x) {
                float row[MS];
                ldv<MS, kStream>(J + i * MS, row);
#pragma unroll
                for (int c = 0; c < MS; ++c)
                    if (UNI || c < y) partial = FADD(partial, FMUL(row[c], buf[c]));
                sum = FADD(sum, partial);
            }
            m[i] = partial;
        }
    }
    if (sum <= 0.0f) sum = 1.0f;
#pragma unroll
    for (int i = 0; i < MS; ++i) m[i] = (UNI || i < x) ? FDIV(m[i], sum) : 0.0f;
}

// buf[i] *= m[i] for i < s unless m[i] is NaN: graph.c:450-459 (combine_message)
template <int MS, bool UNI>
__device__ __forceinline__ void combine(float *buf, const float *m, int s) {
#pragma unroll
    for (int i = 0; i < MS; ++i)
        if ((UNI || i < s) && m[i] == m[i]) buf[i] = FMUL(buf[i], m[i]);
}

// b /= sum(b) over i < s, sum <= 0 replaced by 1 (graph.c:1011-1023)
template <int MS, bool UNI>
__device__ __forceinline__ void normalise(float *b, int s) {
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < MS; ++i)
        if (UNI || i < s) sum = FADD(sum, b[i]);
    if (sum <= 0.0f) sum = 1.0f;
#pragma unroll
    for (int i = 0; i < MS; ++i) b[i] = (UNI || i < s) ? FDIV(b[i], sum) : 0.0f;
}

// ---- block reductions ------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// deterministic: fixed shuffle tree per warp, then warp 0 over warp sums
template <int NT>
__device__ __forceinline__ double block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    if (w == 0) {
        t = lane < NT / 32 ? red[lane] : 0.0;
        t = warp_sum(t);
    }
    __syncthreads();
    return t;  // valid in thread 0
}

}  // namespace bpx

// dispatch on (max states, uniform): instantiates FN<1..10, true/false>
#define BP_DISPATCH_MS(ms, uni, FN, ...)                                              \
    do {                                                                              \
        switch (ms) {                                                                 \
        case 1: return (uni) ? FN<1, true>(__VA_ARGS__) : FN<1, false>(__VA_ARGS__);   \
        case 2: return (uni) ? FN<2, true>(__VA_ARGS__) : FN<2, false>(__VA_ARGS__);   \
        case 3: return (uni) ? FN<3, true>(__VA_ARGS__) : FN<3, false>(__VA_ARGS__);   \
        case 4: return (uni) ? FN<4, true>(__VA_ARGS__) : FN<4, false>(__VA_ARGS__);   \
        case 5: return (uni) ? FN<5, true>(__VA_ARGS__) : FN<5, false>(__VA_ARGS__);   \
        case 6: return (uni) ? FN<6, true>(__VA_ARGS__) : FN<6, false>(__VA_ARGS__);   \
        case 7: return (uni) ? FN<7, true>(__VA_ARGS__) : FN<7, false>(__VA_ARGS__);   \
        case 8: return (uni) ? FN<8, true>(__VA_ARGS__) : FN<8, false>(__VA_ARGS__);   \
        case 9: return (uni) ? FN<9, true>(__VA_ARGS__) : FN<9, false>(__VA_ARGS__);   \
        case 10: return (uni) ? FN<10, true>(__VA_ARGS__) : FN<10, false>(__VA_ARGS__); \
        default: return bpx::set_error(BP_ERR_SHAPE, "state count %u out of range", (unsigned)(ms)); \
        }                                                                             \
    } while (0)
