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

// ---- loads / stores with an L2 eviction-priority policy ------------------
// A policy from createpolicy rides on each access (ld/st .L2::cache_hint);
// it sets the priority of the touched lines only and changes no cache
// configuration.
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

template <int N>
__device__ __forceinline__ void ldv_pol(const float *p, float *o, uint64_t pol) {
    if constexpr (N % 4 == 0) {
#pragma unroll
        for (int k = 0; k < N / 4; ++k)
            asm("ld.global.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                         : "=f"(o[4 * k]), "=f"(o[4 * k + 1]), "=f"(o[4 * k + 2]), "=f"(o[4 * k + 3])
                         : "l"(p + 4 * k), "l"(pol));
    } else if constexpr (N % 2 == 0) {
#pragma unroll
        for (int k = 0; k < N / 2; ++k)
            asm("ld.global.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                         : "=f"(o[2 * k]), "=f"(o[2 * k + 1])
                         : "l"(p + 2 * k), "l"(pol));
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k)
            asm("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(o[k]) : "l"(p + k), "l"(pol));
    }
}

template <int N>
__device__ __forceinline__ void stv_pol(float *p, const float *v, uint64_t pol) {
    if constexpr (N % 4 == 0) {
#pragma unroll
        for (int k = 0; k < N / 4; ++k)
            asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;"
                         :: "l"(p + 4 * k), "f"(v[4 * k]), "f"(v[4 * k + 1]), "f"(v[4 * k + 2]),
                            "f"(v[4 * k + 3]), "l"(pol) : "memory");
    } else if constexpr (N % 2 == 0) {
#pragma unroll
        for (int k = 0; k < N / 2; ++k)
            asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;"
                         :: "l"(p + 2 * k), "f"(v[2 * k]), "f"(v[2 * k + 1]), "l"(pol) : "memory");
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k)
            asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" :: "l"(p + k), "f"(v[k]), "l"(pol) : "memory");
    }
}

// ---- bulk asynchronous copies (global -> shared) and mbarriers -----------
// cp.async.bulk without multicast: the copy engine moves a contiguous range
// into this CTA's shared memory and signals the bytes on an mbarrier.
// Addresses 16-byte aligned, sizes a positive multiple of 16.
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make initialised mbarriers visible to the async proxy
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) accesses
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// one probe of the phase with the given parity (true once it has completed)
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// bounded wait: false when the phase has not completed within `limit_ns`
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
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

// the same send step on a dense x-by-y table (row stride y; for uniform
// graphs y = MS): the operations and their order are send_msg's
template <int MS, bool UNI>
__device__ __forceinline__ void send_msg_dense(const float *__restrict__ J, const float *buf, int x, int y,
                                               float *m) {
    float sum = 0.0f;
#pragma unroll
    for (int i = 0; i < MS; ++i) {
        float partial = 0.0f;
        if (UNI || i < x) {
            float row[MS];
            if constexpr (UNI && MS % 2 == 0) {
                ldv<MS, kReadOnly>(J + i * MS, row);
            } else {
#pragma unroll
                for (int c = 0; c < MS; ++c) row[c] = (UNI || c < y) ? __ldg(J + i * (UNI ? MS : y) + c) : 0.0f;
            }
#pragma unroll
            for (int c = 0; c < MS; ++c)
                if (UNI || c < y) partial = FADD(partial, FMUL(row[c], buf[c]));
            sum = FADD(sum, partial);
        }
        m[i] = partial;
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

// programmatic dependent launch: a kernel launched with the programmatic
// stream-serialization attribute may start before the kernel ahead of it on
// the stream has finished; it must call griddep_wait() before it reads
// anything that kernel (or an earlier one) wrote.  launch_dependents lets the
// next such kernel start once every block of this one has issued it.
__device__ __forceinline__ void griddep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void griddep_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::); }
__device__ __forceinline__ void prefetch_l2(const void *p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

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
