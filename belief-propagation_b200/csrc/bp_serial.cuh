// bp_serial.cuh -- the reference's serial fp32 delta (graph.c:1300-1318)
// decided without forming the serial sum: an interval from the worst-case
// bound on the f64 sum, and a narrow interval from the terms' own rounding
// errors.  Shared by the one-graph loop (loopy.cu) and the batched solver
// (batch.cu).
#pragma once
#include "bp_device.cuh"

namespace bpx {

// The reference's serial fp32 delta (graph.c:1300-1318) decided from an
// interval: for n non-negative terms whose f64 sum is T, the serial sum lies
// within gamma_(n-1) = (n-1)u / (1 - (n-1)u) of the exact sum, u = 2^-24
// (+ 2^-52 for the reference's add through double; Higham, Accuracy and
// Stability of Numerical Algorithms, 2nd ed., section 4.2), plus 2^-149 per
// add for subnormal results; the f64 sum is within 2^-20 of exact for
// n < 2^22.  Directed rounding keeps [lo, hi] safe; +inf when undecidable.
__device__ __forceinline__ void serial_interval(double T, uint64_t n, double &lo, double &hi) {
    const double nd = (double)n;
    const double a = __dmul_ru(nd, 0x1p-24 + 0x1p-52);   // >= (n - 1) u
    if (!(T <= 1.0e300) || a >= 0.25) {
        lo = 0.0;
        hi = __longlong_as_double(0x7ff0000000000000ll);   // +inf: undecided
        return;
    }
    const double gam = __ddiv_ru(a, __dsub_rd(1.0, a));
    const double dT = __dmul_ru(T, 0x1p-20);
    const double S_hi = __dadd_ru(T, dT), S_lo = __dsub_rd(T, dT);
    const double B = __dadd_ru(__dmul_ru(S_hi, gam), __dmul_ru(nd, 0x1p-149));
    lo = fmax(0.0, __dsub_rd(S_lo, B));
    hi = __dadd_ru(S_hi, B);
}

// 1 stop, 0 go on, -1 undecided: s in [lo, hi], previous delta in [plo, phi];
// when both are exact the reference's own float expression decides
__device__ __forceinline__ int serial_decide(double lo, double hi, bool s_exact, double plo, double phi, bool p_exact, float tol) {
    if (s_exact && p_exact) {
        const float s = (float)lo, p = (float)plo;
        return ((s < tol) || (fabsf(FSUB(s, p)) < tol)) ? 1 : 0;
    }
    const double t = (double)tol;
    if (hi < t) return 1;
    // |fl(s - p)| < tol, with s - p in [dlo, dhi] and fl() monotone
    const double dlo = __dsub_rd(lo, phi), dhi = __dsub_ru(hi, plo);
    const double amax = fmax(fabs(dlo), fabs(dhi));
    const double amin = (dlo <= 0.0 && dhi >= 0.0) ? 0.0 : fmin(fabs(dlo), fabs(dhi));
    if (__dadd_ru(__dmul_ru(amax, 1.0 + 0x1p-23), 0x1p-149) < t) return 1;   // fl(x) <= x (1 + 2^-24)
    if (lo >= t && amin >= t) return 0;                                       // tol is a float
    return -1;
}

// ---- a narrow interval for the serial sum, from the terms' own errors ---
//
// s_n = S + sum_k d_k, S = sum t_k exactly, d_k = the rounding error of add k.
// Where the running sum is certainly inside one binade with unit U both
// before and after add k -- judged from the exact prefix P_k and the bound
// |s_k - P_k| <= k u' P_k / (1 - n u') (plus 2^-149 per add) -- the add rounds
// t_k to a multiple of U, so d_k = RN_U(t_k) - t_k is known exactly from t_k
// alone (an exact tie: |d_k| = U / 2, sign unknown).  Elsewhere (the few
// adds next to a binade crossing) |d_k| <= half an ulp of the largest
// possible s_k.  Summing the known d_k and the bounds of the others gives an
// interval about as wide as those few bounds, instead of n u S.

// a block's exclusive scan of doubles (every thread's v); total to all.
// wsum: one double per warp of the block
__device__ __forceinline__ double block_excl_scan_f64(double v, double *wsum, double &total) {
    const int NW = (int)(blockDim.x >> 5);
    const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5;
    double inc = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double o = __shfl_up_sync(0xffffffffu, inc, d);
        if ((int)lane >= d) inc += o;
    }
    if (lane == 31u) wsum[w] = inc;
    __syncthreads();
    double pre = 0.0, tot = 0.0;
    for (int k = 0; k < NW; ++k) {
        const double x = wsum[k];
        if (k < (int)w) pre += x;
        tot += x;
    }
    __syncthreads();   // wsum is free again
    total = tot;
    return pre + inc - v;
}

struct Refine {
    double E;   // sum of the known errors
    double A;   // sum of their magnitudes (for the f64 rounding of E)
    double B;   // sum of the bounds of the unknown ones
    bool bad;   // an inf/NaN term or an overflowing sum: no interval
};

// per-add bound factor: |s_k - P_k| <= P_k k c0 + k 2^-149 (c0 covers
// u' / (1 - n u') and the f64 rounding of P); 0 when n u' is too large
__device__ __forceinline__ double refine_c0(uint64_t n) {
    const double a = __dmul_ru((double)n, 0x1p-24 + 0x1p-52);
    if (a >= 0.25) return 0.0;
    return __dadd_ru(__dmul_ru(__ddiv_ru(0x1p-24 + 0x1p-52, __dsub_rd(1.0, a)), 1.0 + 0x1p-20), 0x1p-51);
}

// one add's contribution: running prefix P before it, t the term, k its
// 1-based index
__device__ __forceinline__ void refine_term(float t, double P, double Pn, uint64_t k, double c0, Refine &r) {
    const uint32_t tb = __float_as_uint(t);
    const uint32_t Et = (tb >> 23) & 0xffu;
    if (Et == 0xffu) {
        r.bad = true;
        return;
    }
    if ((tb & 0x7fffffffu) == 0u || P == 0.0) return;   // adding 0, or onto 0: exact
    const double kd = (double)k;
    const double G = __dadd_ru(__dmul_ru(__dmul_ru(Pn, kd), c0), __dmul_ru(kd, 0x1p-149));
    const double lo = __dsub_rd(P, G), hi = __dadd_ru(Pn, G);
    if (hi >= 0x1p127) {
        r.bad = true;
        return;
    }
    int eu;   // unit exponent of the binade, when certain
    if (hi < 0x1p-126) eu = -149;
    else if (lo >= 0x1p-126 && ilogb(lo) == ilogb(hi)) eu = ilogb(hi) - 23;
    else {
        r.B = __dadd_ru(r.B, hi < 0x1p-126 ? 0x1p-150 : ldexp(1.0, ilogb(hi) - 24));
        return;
    }
    const uint32_t Mt = Et ? ((tb & 0x7fffffu) | 0x800000u) : (tb & 0x7fffffu);
    const int et = Et ? (int)Et - 150 : -149;
    const int shift = et - eu;
    if (Mt == 0u || shift >= 0) return;   // a multiple of U: exact
    const int sh = -shift;
    double d;
    if (sh >= 25) {
        d = -(double)t;   // below U / 2: rounds away entirely
    } else {
        const uint32_t rem = Mt & ((1u << sh) - 1u), half = 1u << (sh - 1);
        if (rem == half) {
            r.B = __dadd_ru(r.B, ldexp(1.0, eu - 1));
            return;
        }
        d = rem > half ? ldexp((double)((1u << sh) - rem), et) : -ldexp((double)rem, et);
    }
    r.E += d;
    r.A += fabs(d);
}

// the terms x[lo, hi) of a sum whose exact prefix before x[lo] is P0, staged
// through buf (cap floats, cap >= 3 threads) in passes of (threads x K)
// terms; every thread of the block (at most NT threads) calls it, and gets
// the block's totals and the end prefix
template <int NT>
__device__ Refine refine_segment(const float *__restrict__ x, uint64_t lo, uint64_t hi, double P0, double c0,
                                 float *buf, uint32_t cap, double &P_end) {
    __shared__ double s_w[NT / 32];
    __shared__ double s_r[4];
    const uint32_t tid = threadIdx.x, nt = blockDim.x, nw = nt >> 5;
    uint32_t K = cap / nt;
    K = (K > 1u ? K - 1u : 1u) & ~1u;
    K = min(max(K, 2u), 30u);
    const uint32_t KS = K + 1u, Pn = nt * K;
    Refine r{0.0, 0.0, 0.0, false};
    double P = P0;
    __syncthreads();   // buf is free
    for (uint64_t base = lo; base < hi; base += Pn) {
        const uint32_t cnt = (uint32_t)min((uint64_t)Pn, hi - base);
        for (uint32_t k = tid; k < cnt; k += nt) buf[(k / K) * KS + k % K] = __ldcg(x + base + k);
        __syncthreads();
        const uint32_t a0 = tid * K, a1 = min(a0 + K, cnt);
        const float *row = buf + tid * KS;
        double ls = 0.0;
        for (uint32_t k = a0; k < a1; ++k) ls += (double)row[k - a0];
        double tot;
        double Pk = P + block_excl_scan_f64(ls, s_w, tot);
        for (uint32_t k = a0; k < a1; ++k) {
            const float t = row[k - a0];
            const double Pn1 = Pk + (double)t;
            refine_term(t, Pk, Pn1, base + k + 1, c0, r);
            Pk = Pn1;
        }
        P += tot;
        __syncthreads();   // buf is rewritten next pass
    }
    // block totals (E, A in any order: their f64 error is bounded by A;
    // B rounded up)
    double e = r.E, a = r.A, b = r.B;
    uint32_t bad = r.bad ? 1u : 0u;
    for (int d = 16; d > 0; d >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, d);
        a += __shfl_xor_sync(0xffffffffu, a, d);
        b = __dadd_ru(b, __shfl_xor_sync(0xffffffffu, b, d));
        bad |= __shfl_xor_sync(0xffffffffu, bad, d);
    }
    __shared__ double s_e[NT / 32], s_a[NT / 32], s_b[NT / 32];
    __shared__ uint32_t s_bad;
    if (tid == 0) s_bad = 0u;
    __syncthreads();
    if ((tid & 31u) == 0u) {
        s_e[tid >> 5] = e;
        s_a[tid >> 5] = a;
        s_b[tid >> 5] = b;
        if (bad) s_bad = 1u;
    }
    __syncthreads();
    if (tid == 0) {
        double E = 0.0, A = 0.0, B = 0.0;
        for (uint32_t w = 0; w < nw; ++w) {
            E += s_e[w];
            A += s_a[w];
            B = __dadd_ru(B, s_b[w]);
        }
        s_r[0] = E;
        s_r[1] = A;
        s_r[2] = B;
        s_r[3] = s_bad ? 1.0 : 0.0;
    }
    __syncthreads();
    Refine out{s_r[0], s_r[1], s_r[2], s_r[3] != 0.0};
    P_end = P;
    __syncthreads();
    return out;
}

// the interval of s from the exact-sum estimate T (an f64 sum of n terms),
// the known errors E (magnitudes A) and the bounds B
__device__ __forceinline__ void refine_interval(double T, const Refine &r, uint64_t n, double &lo, double &hi) {
    const double m = (double)n + 0x1p21;   // adds in any f64 summation of the pieces
    const double tS = __dmul_ru(__dmul_ru(T, m), 0x1p-52), tE = __dmul_ru(__dmul_ru(r.A, m), 0x1p-52);
    const double w = __dadd_ru(__dadd_ru(tS, tE), __dmul_ru(r.B, 1.0 + 0x1p-40));
    const double mid = T + r.E;
    const double mw = __dmul_ru(fabs(mid), 0x1p-52);   // the rounding of mid
    lo = fmax(0.0, __dsub_rd(__dsub_rd(mid, mw), w));
    hi = __dadd_ru(__dadd_ru(mid, mw), w);
}

// a block's narrowed interval of the serial sum of x[0, n); false if none
template <int NT>
__device__ __noinline__ bool refine_block(const float *x, uint64_t n, float *buf, uint32_t cap, double &lo, double &hi) {
    const double c0 = refine_c0(n);
    if (c0 == 0.0) return false;
    double T;
    const Refine r = refine_segment<NT>(x, 0, n, 0.0, c0, buf, cap, T);
    if (r.bad) return false;
    refine_interval(T, r, n, lo, hi);
    return true;
}

// [lo, hi] holding one float only: that float
__device__ __forceinline__ bool interval_pins(double lo, double hi, float &f) {
    const float a = __double2float_ru(lo), b = __double2float_rd(hi);
    f = a;
    return a == b;
}

}  // namespace bpx
