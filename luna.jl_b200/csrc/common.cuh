// Shared definitions for the sm_100a UPPE kernels: complex arithmetic, the buffer
// swizzle and the twiddle tables.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#ifndef LUNA_BLOCK
#define LUNA_BLOCK 512
#endif
#ifndef LUNA_WARPS
#define LUNA_WARPS (LUNA_BLOCK / 32)
#endif

namespace luna {

template <typename R> struct alignas(2 * sizeof(R)) cpx { R x, y; };

template <typename R> __host__ __device__ __forceinline__ cpx<R> mk(R a, R b) { cpx<R> c; c.x = a; c.y = b; return c; }
template <typename R> __device__ __forceinline__ cpx<R> operator+(cpx<R> a, cpx<R> b) { return mk<R>(a.x + b.x, a.y + b.y); }
template <typename R> __device__ __forceinline__ cpx<R> operator-(cpx<R> a, cpx<R> b) { return mk<R>(a.x - b.x, a.y - b.y); }
template <typename R> __device__ __forceinline__ cpx<R> operator*(cpx<R> a, cpx<R> b) {
    return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename R> __device__ __forceinline__ cpx<R> scale(R s, cpx<R> a) { return mk<R>(s * a.x, s * a.y); }
template <typename R> __device__ __forceinline__ cpx<R> conj(cpx<R> a) { return mk<R>(a.x, -a.y); }
template <typename R> __device__ __forceinline__ R abs2(cpx<R> a) { return a.x * a.x + a.y * a.y; }
// multiply by -i (forward transform) or +i (inverse transform)
template <typename R, bool INV> __device__ __forceinline__ cpx<R> mul_mi(cpx<R> a) {
    return INV ? mk<R>(-a.y, a.x) : mk<R>(a.y, -a.x);
}
template <typename Rt, typename R> __device__ __forceinline__ cpx<Rt> cvt(cpx<R> a) {
    return mk<Rt>((Rt)a.x, (Rt)a.y);
}

__device__ __forceinline__ cpx<double> ldg(const cpx<double>* p) {
    double2 v = __ldg(reinterpret_cast<const double2*>(p));
    return mk<double>(v.x, v.y);
}
__device__ __forceinline__ cpx<float> ldg(const cpx<float>* p) {
    float2 v = __ldg(reinterpret_cast<const float2*>(p));
    return mk<float>(v.x, v.y);
}

// Buffer swizzle: XOR the low index bits of each 128-byte row with two higher bit
// fields, so that the strided Stockham writes of the first passes and the contiguous
// reads both spread over the 32 shared-memory banks. It permutes elements only inside
// aligned groups of 8 (FP64 complex) or 16 (FP32 complex), so warp-contiguous accesses
// to a swizzled buffer in global memory stay fully coalesced.
template <typename R> struct Swz;
template <> struct Swz<double> {
    static __device__ __forceinline__ int f(int i) { return i ^ ((i >> 3) & 7) ^ ((i >> 6) & 7); }
};
template <> struct Swz<float> {
    static __device__ __forceinline__ int f(int i) { return i ^ ((i >> 4) & 15) ^ ((i >> 8) & 15); }
};

// Twiddle factors exp(-2*pi*i*a/TW_MMAX) are the product hi[a >> 6] * lo[a & 63] of two
// small tables; TW_MMAX bounds every transform length handled here.
#define TW_LOG_MMAX 17
#define TW_MMAX (1 << TW_LOG_MMAX)
#define TW_NLO 64
#define TW_NHI (TW_MMAX / TW_NLO)

template <typename R> struct TwTab {
    const cpx<R>* lo;
    const cpx<R>* hi;
};

// exp(-2*pi*i*a/TW_MMAX), conjugated for inverse transforms
template <typename R, bool INV>
__device__ __forceinline__ cpx<R> twiddle(const TwTab<R>& tw, unsigned a) {
    a &= (TW_MMAX - 1);
    cpx<R> w = ldg(tw.hi + (a >> 6)) * ldg(tw.lo + (a & 63));
    return INV ? conj(w) : w;
}

// Status codes shared with the C ABI (include/luna_b200.h)
enum {
    ST_OK = 0,
    ST_FIELD_ABOVE_EMAX = 1,
    ST_REPEAT_LIMIT = 2,
    ST_NONFINITE = 3,
    ST_STEP_BUDGET = 4,
    ST_WAIT_TIMEOUT = 5,  // a bounded device-side wait (tensor-core completion) ran out
};

}  // namespace luna
