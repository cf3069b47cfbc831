// Block-wide FFT for one CTA of LUNA_BLOCK threads, in place in shared or global memory.
//
// A length-M transform is split as M = P * Mb with Mb <= EMAX * LUNA_BLOCK (EMAX = 8
// complex values per thread; with 16 for FP32 the butterflies spill registers and the
// solver steps are ~20 % slower on B200). The P sub-transforms of length Mb are
// Stockham passes done in place: every thread loads its E = Mb/LUNA_BLOCK inputs,
// synchronises, computes its radix-R butterflies and writes the outputs back.
// One radix-P pass joins the sub-transforms:
//   * inverse transforms run decimation-in-frequency: natural-order input, radix-P pass,
//     sub-transforms; the result is in the "split" order  X[P*k + p] at p*Mb + k;
//   * forward transforms run decimation-in-time: split-order input (element n at
//     (n mod P)*Mb + n/P), sub-transforms, radix-P pass; the result is in natural order.
// An inverse transform followed by pointwise work in place and a forward transform thus
// never needs a reordering pass. For P == 1 both orders are the natural order.
//
// Stockham pass with radix R and span L: butterfly j, k = j mod L, inputs x[j + r*Mb/R],
// twiddle exp(-+2*pi*i*r*k/(L*R)), R-point DFT, outputs y[(j-k)*R + k + r*L].
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
    const R c = (R)(Q <= 8 ? cos16(Q) : -cos16(16 - Q));
    const R s = (R)(Q <= 8 ? cos16(8 - Q) : cos16(Q - 8));
    // forward: b * (c - i s); inverse: b * (c + i s)
    return INV ? mk<R>(b.x * c - b.y * s, b.x * s + b.y * c)
               : mk<R>(b.x * c + b.y * s, b.y * c - b.x * s);
}

template <int N> __host__ __device__ constexpr int ilog2c() { return N <= 1 ? 0 : 1 + ilog2c<N / 2>(); }

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

// In-register RAD-point DFT (radix-2 decimation-in-time network): the inputs must sit in
// bit-reversed order (v[i] = x[bitrev(i)]); the outputs come out in natural order.
template <typename R, bool INV, int RAD>
__device__ __forceinline__ void dft_br(cpx<R>* v) {
    bfly_stages<R, INV, RAD, 1>(v);
}

template <typename R>
struct FftEmax { static constexpr int v = 8; };

// largest transform held by one CTA: P <= 8 sub-transforms of EMAX*LUNA_BLOCK
template <typename R>
struct FftMmax { static constexpr int v = 8 * FftEmax<R>::v * LUNA_BLOCK; };

__device__ __forceinline__ int ilog2i(unsigned x) { return 31 - __clz(x); }

// Multiply v[i] (bit-reversed slot i holds input r = bitrev(i)) by w^r for r = 1..RAD-1.
// w comes from one table lookup; w^r is a product of the binary powers w, w^2, w^4, ...
template <typename R, int RAD>
__device__ __forceinline__ void apply_twiddles(cpx<R>* v, cpx<R> w) {
    constexpr int NB = ilog2c<RAD>();
    cpx<R> wb[NB > 0 ? NB : 1];
    wb[0] = w;
#pragma unroll
    for (int b = 1; b < NB; ++b) wb[b] = wb[b - 1] * wb[b - 1];
#pragma unroll
    for (int i = 1; i < RAD; ++i) {
        const int r = bitrev<RAD>(i);
        cpx<R> f;
        bool have = false;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            if (r & (1 << b)) {
                f = have ? f * wb[b] : wb[b];
                have = true;
            }
        }
        v[i] = v[i] * f;
    }
}

// One in-place Stockham pass over a sub-transform of length Mb at `buf`; nact threads
// are active, each with E/RAD butterflies.
template <typename R, bool INV, int E, int RAD>
__device__ __forceinline__ void pass_inplace(cpx<R>* buf, int Mb, int L, int nact, const TwTab<R>& tw) {
    const int t = threadIdx.x;
    constexpr int NB = E / RAD;
    cpx<R> v[E];
    const int stride = Mb / RAD;
    if (t < nact) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + b * nact;
#pragma unroll
            for (int i = 0; i < RAD; ++i) v[b * RAD + i] = buf[Swz<R>::f(j + bitrev<RAD>(i) * stride)];
        }
    }
    __syncthreads();
    if (t < nact) {
        const int shift = TW_LOG_MMAX - ilog2i((unsigned)(L * RAD));
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + b * nact;
            const int k = j & (L - 1);
            if (L > 1) apply_twiddles<R, RAD>(&v[b * RAD], twiddle<R, INV>(tw, (unsigned)k << shift));
            dft_br<R, INV, RAD>(&v[b * RAD]);
            const int base = (j - k) * RAD + k;
#pragma unroll
            for (int r = 0; r < RAD; ++r) buf[Swz<R>::f(base + r * L)] = v[b * RAD + r];
        }
    }
    __syncthreads();
}

// In-place Stockham transform of one sub-block of length Mb = E * nact: a twiddle-free
// first pass of the remainder radix, then passes of radix E.
template <typename R, bool INV, int E>
__device__ __forceinline__ void sub_fft(cpx<R>* buf, int Mb, const TwTab<R>& tw) {
    constexpr int LR = ilog2c<E>();
    const int nact = Mb / E;
    const int rem = ilog2i((unsigned)Mb) % LR;
    int L = 1;
    if (rem != 0) {
        const int r0 = 1 << rem;
        if constexpr (E > 2) { if (r0 == 2) pass_inplace<R, INV, E, 2>(buf, Mb, 1, nact, tw); }
        if constexpr (E > 4) { if (r0 == 4) pass_inplace<R, INV, E, 4>(buf, Mb, 1, nact, tw); }
        if constexpr (E > 8) { if (r0 == 8) pass_inplace<R, INV, E, 8>(buf, Mb, 1, nact, tw); }
        L = r0;
    }
    while (L < Mb) {
        pass_inplace<R, INV, E, E>(buf, Mb, L, nact, tw);
        L *= E;
    }
}

// The same transform of two buffers at once: one pass processes both, so the two
// transforms share their barriers and twiddles (E/RAD butterflies per buffer and thread).
template <typename R, bool INV, int E, int RAD>
__device__ __forceinline__ void pass_inplace2(cpx<R>* ba, cpx<R>* bb, int Mb, int L, int nact, const TwTab<R>& tw) {
    const int t = threadIdx.x;
    constexpr int NB = E / RAD;
    cpx<R> va[E], vb[E];
    const int stride = Mb / RAD;
    if (t < nact) {
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int j = t + b * nact;
#pragma unroll
            for (int i = 0; i < RAD; ++i) {
                const int a = Swz<R>::f(j + bitrev<RAD>(i) * stride);
                va[b * RAD + i] = ba[a];
                vb[b * RAD + i] = bb[a];
            }
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
                const cpx<R> w = twiddle<R, INV>(tw, (unsigned)k << shift);
                apply_twiddles<R, RAD>(&va[b * RAD], w);
                apply_twiddles<R, RAD>(&vb[b * RAD], w);
            }
            dft_br<R, INV, RAD>(&va[b * RAD]);
            dft_br<R, INV, RAD>(&vb[b * RAD]);
            const int base = (j - k) * RAD + k;
#pragma unroll
            for (int r = 0; r < RAD; ++r) {
                const int a = Swz<R>::f(base + r * L);
                ba[a] = va[b * RAD + r];
                bb[a] = vb[b * RAD + r];
            }
        }
    }
    __syncthreads();
}

template <typename R, bool INV, int E>
__device__ __forceinline__ void sub_fft2(cpx<R>* ba, cpx<R>* bb, int Mb, const TwTab<R>& tw) {
    constexpr int LR = ilog2c<E>();
    const int nact = Mb / E;
    const int rem = ilog2i((unsigned)Mb) % LR;
    int L = 1;
    if (rem != 0) {
        const int r0 = 1 << rem;
        if constexpr (E > 2) { if (r0 == 2) pass_inplace2<R, INV, E, 2>(ba, bb, Mb, 1, nact, tw); }
        if constexpr (E > 4) { if (r0 == 4) pass_inplace2<R, INV, E, 4>(ba, bb, Mb, 1, nact, tw); }
        L = r0;
    }
    while (L < Mb) {
        pass_inplace2<R, INV, E, E>(ba, bb, Mb, L, nact, tw);
        L *= E;
    }
}

// Radix-P pass joining the sub-transforms, in place (each thread owns the P elements
// k + q*Mb). DIT (forward): X[k + q*Mb] = sum_p W_P^{pq} * (W_M^{pk} * A_p[k]).
// DIF (inverse):           b_p[k] = W_M^{-pk} * sum_q W_P^{-pq} * x[k + q*Mb].
template <typename R, bool INV, int P>
__device__ __forceinline__ void join_pass(cpx<R>* buf, int M, const TwTab<R>& tw) {
    const int Mb = M / P;
    const int shift = TW_LOG_MMAX - ilog2i((unsigned)M);
    __syncthreads();
    for (int k = threadIdx.x; k < Mb; k += LUNA_BLOCK) {
        cpx<R> v[P];
#pragma unroll
        for (int i = 0; i < P; ++i) v[i] = buf[Swz<R>::f(k + bitrev<P>(i) * Mb)];
        if (!INV) {
            apply_twiddles<R, P>(v, twiddle<R, INV>(tw, (unsigned)k << shift));
            dft_br<R, INV, P>(v);
        } else {
            dft_br<R, INV, P>(v);
            // v[p] = sum_q W_P^{-pq} x_q; apply W_M^{-pk}
            const cpx<R> w = twiddle<R, INV>(tw, (unsigned)k << shift);
            cpx<R> f = w;
#pragma unroll
            for (int p = 1; p < P; ++p) {
                v[p] = v[p] * f;
                f = f * w;
            }
        }
#pragma unroll
        for (int q = 0; q < P; ++q) buf[Swz<R>::f(k + q * Mb)] = v[q];
    }
    __syncthreads();
}

template <typename R, bool INV>
__device__ __forceinline__ void sub_ffts(cpx<R>* buf, int M, int P, const TwTab<R>& tw) {
    const int Mb = M / P;
    int E = Mb / LUNA_BLOCK;
    if (E < 2) E = 2;
    for (int p = 0; p < P; ++p) {
        cpx<R>* b = buf + (size_t)p * Mb;
        if (E == 2) sub_fft<R, INV, 2>(b, Mb, tw);
        else if (E == 4) sub_fft<R, INV, 4>(b, Mb, tw);
        else if (E == 8) sub_fft<R, INV, 8>(b, Mb, tw);
        else if constexpr (FftEmax<R>::v >= 16) sub_fft<R, INV, 16>(b, Mb, tw);
    }
}

// Out-of-place Stockham pass (natural order in and out) between two global-memory buffers;
// used when a transform does not fit in shared memory and a second buffer is available.
// Each butterfly's twiddles come from independent table lookups (no dependent chain), which
// keeps more L2 requests in flight than the binary-power form used in shared memory.
template <typename R, bool INV, int RAD>
__device__ __forceinline__ void pass_oop(const cpx<R>* src, cpx<R>* dst, int M, int L, const TwTab<R>& tw) {
    const int stride = M / RAD;
    const int shift = TW_LOG_MMAX - ilog2i((unsigned)(L * RAD));
    for (int j = threadIdx.x; j < stride; j += LUNA_BLOCK) {
        cpx<R> v[RAD];
#pragma unroll
        for (int i = 0; i < RAD; ++i) v[i] = src[Swz<R>::f(j + bitrev<RAD>(i) * stride)];
        const int k = j & (L - 1);
        if (L > 1) {
#pragma unroll
            for (int i = 1; i < RAD; ++i)
                v[i] = v[i] * twiddle<R, INV>(tw, (unsigned)(bitrev<RAD>(i) * k) << shift);
        }
        dft_br<R, INV, RAD>(v);
        const int base = (j - k) * RAD + k;
#pragma unroll
        for (int r = 0; r < RAD; ++r) dst[Swz<R>::f(base + r * L)] = v[r];
    }
    __syncthreads();
}

// Natural-order out-of-place transform with radix-16 passes (the last one takes the
// remainder radix); returns the buffer holding the result (a or b).
template <typename R, bool INV>
__device__ __forceinline__ cpx<R>* fft_oop(cpx<R>* a, cpx<R>* b, int M, const TwTab<R>& tw) {
    int L = 1;
    cpx<R>* src = a;
    cpx<R>* dst = b;
    while (L < M) {
        const int rad = min(16, M / L);
        if (rad == 2) pass_oop<R, INV, 2>(src, dst, M, L, tw);
        else if (rad == 4) pass_oop<R, INV, 4>(src, dst, M, L, tw);
        else if (rad == 8) pass_oop<R, INV, 8>(src, dst, M, L, tw);
        else pass_oop<R, INV, 16>(src, dst, M, L, tw);
        cpx<R>* t = src;
        src = dst;
        dst = t;
        L *= rad;
    }
    return src;
}

// number of sub-transforms for a length-M transform
template <typename R>
__host__ __device__ __forceinline__ int fft_nsplit(int M) {
    int P = 1;
    while (M / P > FftEmax<R>::v * LUNA_BLOCK) P *= 2;
    return P;
}

// Position of element n of a split-order array of length M with P sub-transforms.
__device__ __forceinline__ int split_pos(int n, int M, int P) {
    return (n & (P - 1)) * (M / P) + n / P;
}

// Unnormalised DFT of length M (power of two, 2 <= M <= FftMmax).
// With alt == nullptr (shared-memory buffers) it runs in place:
//   forward (INV=false): split-order input -> natural-order output
//   inverse (INV=true):  natural-order input -> split-order output
// With a second buffer alt (global-memory buffers) it runs out of place in natural order
// both ways. Returns the buffer holding the result. The caller synchronises before the
// call (the input is written by other threads); the call ends with a barrier.
template <typename R, bool INV>
__device__ __forceinline__ void block_fft_split(cpx<R>* buf, int M, const TwTab<R>& tw);

template <typename R, bool INV>
__device__ __noinline__ cpx<R>* block_fft(cpx<R>* buf, cpx<R>* alt, int M, const TwTab<R>& tw) {
    if (alt) return fft_oop<R, INV>(buf, alt, M, tw);
    block_fft_split<R, INV>(buf, M, tw);
    return buf;
}

// split factor of a length-M transform on a buffer (1: natural order, out of place)
template <typename R>
__device__ __forceinline__ int buf_split(const cpx<R>* alt, int M) {
    return alt ? 1 : fft_nsplit<R>(M);
}

template <typename R, bool INV>
__device__ __forceinline__ void block_fft_split(cpx<R>* buf, int M, const TwTab<R>& tw) {
    const int P = fft_nsplit<R>(M);
    if (INV) {
        if (P == 2) join_pass<R, INV, 2>(buf, M, tw);
        else if (P == 4) join_pass<R, INV, 4>(buf, M, tw);
        else if (P == 8) join_pass<R, INV, 8>(buf, M, tw);
        sub_ffts<R, INV>(buf, M, P, tw);
    } else {
        sub_ffts<R, INV>(buf, M, P, tw);
        if (P == 2) join_pass<R, INV, 2>(buf, M, tw);
        else if (P == 4) join_pass<R, INV, 4>(buf, M, tw);
        else if (P == 8) join_pass<R, INV, 8>(buf, M, tw);
    }
}

}  // namespace luna
