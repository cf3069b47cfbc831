// Block-wide Stockham FFT for one CTA of LUNA_BLOCK threads.
//
// Two forms:
//  * in-place: every active thread holds E = M/nact elements in registers, so each
//    radix-R pass reads all of its inputs, synchronises, and writes its outputs back
//    to the same (swizzled) buffer. Used whenever E <= EMAX (16 for FP64, 32 for FP32);
//    this is the shared-memory path.
//  * out-of-place: ping-pongs between two swizzled buffers (used for transforms too
//    large to hold in registers, which then live in L2-resident global scratch).
//
// Pass p with radix R and span L (product of the earlier radices) maps butterfly j,
// k = j mod L, inputs x[j + r*M/R] -> twiddle exp(-+2*pi*i*r*k/(L*R)) -> R-point DFT ->
// outputs y[(j-k)*R + k + r*L]; after the last pass the data is in natural order.
#pragma once
#include "common.cuh"

namespace luna {

// cos(pi*q/16) for q = 0..8; used for the in-register DFT twiddles (q/32 turns)
__device__ __forceinline__ double cos16(int q) {
    switch (q) {
        case 0: return 1.0;
        case 1: return 0.9807852804032304;
        case 2: return 0.9238795325112867;
        case 3: return 0.8314696123025452;
        case 4: return 0.7071067811865476;
        case 5: return 0.5555702330196023;
        case 6: return 0.38268343236508984;
        case 7: return 0.19509032201612833;
        default: return 0.0;
    }
}

// multiply by exp(-+2*pi*i*q/32), q in [0, 16)
template <typename R, bool INV, int Q>
__device__ __forceinline__ cpx<R> rot32(cpx<R> b) {
    if (Q == 0) return b;
    if (Q == 8) return mul_mi<R, INV>(b);
    // cos/sin of 2*pi*Q/32 = pi*Q/16
    const R c = (R)(Q <= 8 ? cos16(Q) : -cos16(16 - Q));
    const R s = (R)(Q <= 8 ? cos16(8 - Q) : cos16(Q - 8));
    // forward: b * (c - i s); inverse: b * (c + i s)
    return INV ? mk<R>(b.x * c - b.y * s, b.x * s + b.y * c)
               : mk<R>(b.x * c + b.y * s, b.y * c - b.x * s);
}

template <int RAD>
__host__ __device__ constexpr int bitrev(int i) {
    int r = 0;
    for (int b = 1; b < RAD; b <<= 1) {
        r = (r << 1) | (i & 1);
        i >>= 1;
    }
    return r;
}

template <typename R, bool INV, int RAD, int S, int K, int J>
__device__ __forceinline__ void bfly_step(cpx<R>* v) {
    if constexpr (J < S) {
        cpx<R> a = v[K + J];
        cpx<R> b = rot32<R, INV, J * (32 / (2 * S))>(v[K + J + S]);
        v[K + J] = a + b;
        v[K + J + S] = a - b;
        bfly_step<R, INV, RAD, S, K, J + 1>(v);
    }
}

template <typename R, bool INV, int RAD, int S, int K>
__device__ __forceinline__ void bfly_group(cpx<R>* v) {
    if constexpr (K < RAD) {
        bfly_step<R, INV, RAD, S, K, 0>(v);
        bfly_group<R, INV, RAD, S, K + 2 * S>(v);
    }
}

template <typename R, bool INV, int RAD, int S>
__device__ __forceinline__ void bfly_stages(cpx<R>* v) {
    if constexpr (S < RAD) {
        bfly_group<R, INV, RAD, S, 0>(v);
        bfly_stages<R, INV, RAD, 2 * S>(v);
    }
}

// in-register RAD-point DFT, natural order in and out (radix-2 DIT network)
template <typename R, bool INV, int RAD>
__device__ __forceinline__ void dft(cpx<R>* u) {
    cpx<R> v[RAD];
#pragma unroll
    for (int i = 0; i < RAD; ++i) v[i] = u[bitrev<RAD>(i)];
    bfly_stages<R, INV, RAD, 1>(v);
#pragma unroll
    for (int i = 0; i < RAD; ++i) u[i] = v[i];
}

template <typename R>
struct FftEmax { static constexpr int v = (sizeof(R) == 8) ? 16 : 32; };

template <int N> __host__ __device__ constexpr int ilog2c() { return N <= 1 ? 0 : 1 + ilog2c<N / 2>(); }

__device__ __forceinline__ int ilog2i(unsigned x) { return 31 - __clz(x); }

// One in-place pass: nact active threads, each with E/RAD butterflies.
template <typename R, bool INV, int E, int RAD>
__device__ __forceinline__ void pass_inplace(cpx<R>* buf, int M, int L, int nact, const TwTab<R>& tw) {
    const int t = threadIdx.x;
    constexpr int NB = E / RAD;
    cpx<R> v[E];
    const int stride = M / RAD;
    if (t < nact) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + b * nact;
#pragma unroll
            for (int r = 0; r < RAD; ++r) v[b * RAD + r] = buf[Swz<R>::f(j + r * stride)];
        }
    }
    __syncthreads();
    if (t < nact) {
        const int shift = TW_LOG_MMAX - ilog2i((unsigned)(L * RAD));
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + b * nact;
            const int k = j & (L - 1);
            if (L > 1) {
#pragma unroll
                for (int r = 1; r < RAD; ++r)
                    v[b * RAD + r] = v[b * RAD + r] * twiddle<R, INV>(tw, (unsigned)(r * k) << shift);
            }
            dft<R, INV, RAD>(&v[b * RAD]);
            const int base = (j - k) * RAD + k;
#pragma unroll
            for (int r = 0; r < RAD; ++r) buf[Swz<R>::f(base + r * L)] = v[b * RAD + r];
        }
    }
    __syncthreads();
}

template <typename R, bool INV, int E>
__device__ void fft_inplace(cpx<R>* buf, int M, const TwTab<R>& tw) {
    const int nact = M / E;
    int L = 1;
    while (L < M) {
        const int rad = min(E, M / L);
        if constexpr (E >= 2) if (rad == 2) pass_inplace<R, INV, E, 2>(buf, M, L, nact, tw);
        if constexpr (E >= 4) if (rad == 4) pass_inplace<R, INV, E, 4>(buf, M, L, nact, tw);
        if constexpr (E >= 8) if (rad == 8) pass_inplace<R, INV, E, 8>(buf, M, L, nact, tw);
        if constexpr (E >= 16) if (rad == 16) pass_inplace<R, INV, E, 16>(buf, M, L, nact, tw);
        if constexpr (E >= 32) if (rad == 32) pass_inplace<R, INV, E, 32>(buf, M, L, nact, tw);
        L *= rad;
    }
}

template <typename R, bool INV, int RAD>
__device__ __forceinline__ void pass_oop(const cpx<R>* src, cpx<R>* dst, int M, int L, const TwTab<R>& tw) {
    const int stride = M / RAD;
    const int shift = TW_LOG_MMAX - ilog2i((unsigned)(L * RAD));
    for (int j = threadIdx.x; j < stride; j += LUNA_BLOCK) {
        cpx<R> v[RAD];
#pragma unroll
        for (int r = 0; r < RAD; ++r) v[r] = src[Swz<R>::f(j + r * stride)];
        const int k = j & (L - 1);
        if (L > 1) {
#pragma unroll
            for (int r = 1; r < RAD; ++r) v[r] = v[r] * twiddle<R, INV>(tw, (unsigned)(r * k) << shift);
        }
        dft<R, INV, RAD>(v);
        const int base = (j - k) * RAD + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) dst[Swz<R>::f(base + r * L)] = v[r];
    }
    __syncthreads();
}

// returns the buffer holding the result (a or b)
template <typename R, bool INV>
__device__ cpx<R>* fft_oop(cpx<R>* a, cpx<R>* b, int M, const TwTab<R>& tw) {
    int L = 1;
    cpx<R>* src = a;
    cpx<R>* dst = b;
    while (L < M) {
        const int rad = min(16, M / L);
        if (rad == 2) pass_oop<R, INV, 2>(src, dst, M, L, tw);
        else if (rad == 4) pass_oop<R, INV, 4>(src, dst, M, L, tw);
        else if (rad == 8) pass_oop<R, INV, 8>(src, dst, M, L, tw);
        else pass_oop<R, INV, 16>(src, dst, M, L, tw);
        cpx<R>* tmp = src;
        src = dst;
        dst = tmp;
        L *= rad;
    }
    return src;
}

// Whether a length-M transform runs in place (registers) for this block size.
template <typename R>
__device__ __forceinline__ bool fft_is_inplace(int M) {
    int E = M / LUNA_BLOCK;
    return E <= FftEmax<R>::v;
}

// Unnormalised DFT (forward, exp(-...)) or inverse (exp(+...)) of length M (power of two,
// 2 <= M <= TW_MMAX). Returns the buffer that holds the result: `buf` for in-place
// transforms, otherwise `buf` or `alt`.
template <typename R, bool INV>
__device__ cpx<R>* block_fft(cpx<R>* buf, cpx<R>* alt, int M, const TwTab<R>& tw) {
    int E = M / LUNA_BLOCK;
    if (E < 2) E = 2;
    if (E == 2) { fft_inplace<R, INV, 2>(buf, M, tw); return buf; }
    if (E == 4) { fft_inplace<R, INV, 4>(buf, M, tw); return buf; }
    if (E == 8) { fft_inplace<R, INV, 8>(buf, M, tw); return buf; }
    if (E == 16) { fft_inplace<R, INV, 16>(buf, M, tw); return buf; }
    if constexpr (FftEmax<R>::v >= 32) {
        if (E == 32) { fft_inplace<R, INV, 32>(buf, M, tw); return buf; }
    }
    return fft_oop<R, INV>(buf, alt, M, tw);
}

}  // namespace luna
