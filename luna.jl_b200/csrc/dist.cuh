// Distributed solver: one mode-averaged instance integrated by a thread-block cluster of
// R CTAs (DIST_R, or DIST_R_BIG for the longest instances), for the long instances of a
// batch (field-resolved grid, FP64 or mixed precision).
//
// The RK45 loop, stage combinations, error norm and controller are those of
// solve_instance; what is split is every per-bin and per-sample loop and every transform:
//   * frequency bins: CTA p owns the bins n = p (mod R) of every Nw-vector (stage inputs and
//     derivatives, exp(L dz), the window filter, the saves), so no global array is shared
//     between CTAs;
//   * time samples: CTA q holds the contiguous block of sample pairs m in [q Mb, (q+1) Mb)
//     (Mb = M/R, M = No/2), so the plasma integrals run as block scans with carries;
//   * transforms of length M = R Mb: the inverse one is decimation in time (CTA p transforms
//     the bins R k + p, then the blocks are joined by a radix-R step), the forward one
//     decimation in frequency (radix-R step, then CTA p transforms its sub-sequence), both
//     on Mb-point Stockham sub-transforms in shared memory;
//   * the Raman convolution (a 2M-point transform) on 2R sub-transforms, CTA c holding
//     the pair {c, 2R - c} ({0, R} for c = 0) so that the real-transform split pairs k with
//     2M - k inside one CTA.
// Data cross between CTAs only through distributed shared memory (ld.shared::cluster) after
// cluster barriers; every CTA takes the same barriers in the same order (the controller
// runs in every CTA on identical, identically summed inputs).
#pragma once
#include <cooperative_groups.h>

#include "uppe.cuh"

namespace luna {

// cluster sizes: DIST_R CTAs per distributed instance, DIST_R_BIG for the longest ones
// (non-portable clusters); the device code is templated on the size R
#define DIST_R 8
#define DIST_R_BIG 16
// elements per thread whose remote loads are issued together
template <int R>
struct DUnr {
    static constexpr int v = 16 / R > 0 ? 16 / R : 1;
    static constexpr int raman = 8 / R > 0 ? 8 / R : 1;
};

namespace dcg = cooperative_groups;

template <typename Rl>
struct DWs {
    double* red;   // 3 * LUNA_WARPS block-reduction scratch
    double* tot;   // 3 * LUNA_WARPS scan totals
    int* flag;     // status bits raised by the responses
    double* xs;    // [16] values this CTA publishes to the cluster
    TwTab<Rl> tw;
    cpx<Rl>* stg;  // [Mb + 16] own bins of the spectrum; plasma rates
    cpx<Rl>* fb;   // [Mb] this CTA's sub-transform; plasma ionisation fractions
    cpx<Rl>* tb;   // [Mb] this CTA's block of time-domain sample pairs
    cpx<Rl>* ef;   // [Mb + 16] exp(L dz) of the own bins
    cpx<Rl>* rb0;  // [Mb] Raman sub-transforms
    cpx<Rl>* rb1;  // [Mb]
    int rank;
};

__host__ __device__ inline size_t dist_smem_bytes(int No, size_t csize, int R = DIST_R) {
    const size_t Mb = (size_t)(No / 2) / R;
    return LUNA_SMALL_BYTES + 2 * align_up((Mb + 16) * csize, 256) + 4 * align_up(Mb * csize, 256);
}

template <typename Rl, int R>
__device__ void plan_dws(const LunaInst& I, char* smem, DWs<Rl>& d, const TwTab<Rl>& tw, int rank) {
    d.red = reinterpret_cast<double*>(smem);
    d.tot = d.red + 3 * LUNA_WARPS;
    d.flag = reinterpret_cast<int*>(d.tot + 3 * LUNA_WARPS);
    d.xs = reinterpret_cast<double*>(smem + 1024);
    d.tw = tw;
    d.rank = rank;
    const size_t c = sizeof(cpx<Rl>);
    const size_t Mb = (size_t)(I.No / 2) / R;
    const size_t bs = align_up((Mb + 16) * c, 256), bm = align_up(Mb * c, 256);
    size_t off = LUNA_SMALL_BYTES;
    d.stg = reinterpret_cast<cpx<Rl>*>(smem + off);
    off += bs;
    d.ef = reinterpret_cast<cpx<Rl>*>(smem + off);
    off += bs;
    d.fb = reinterpret_cast<cpx<Rl>*>(smem + off);
    off += bm;
    d.tb = reinterpret_cast<cpx<Rl>*>(smem + off);
    off += bm;
    d.rb0 = reinterpret_cast<cpx<Rl>*>(smem + off);
    off += bm;
    d.rb1 = reinterpret_cast<cpx<Rl>*>(smem + off);
}

__device__ __forceinline__ void dsync() { dcg::this_cluster().sync(); }

template <typename T>
__device__ __forceinline__ T* drem(T* p, int r) {
    return dcg::this_cluster().map_shared_rank(p, r);
}

// In-place Stockham transform (natural order in and out) of one buffer of length Mb, in
// radix-8 passes (Mb/8 threads active): fewer barrier-separated passes matter more than
// the idle threads for the short sub-transforms of a cluster.
template <typename Rl, bool INV>
__device__ __forceinline__ void sub_fft_any(cpx<Rl>* b, int Mb, const TwTab<Rl>& tw) {
    sub_fft<Rl, INV, 8>(b, Mb, tw);
}

// exp(-+2 pi i a / 2^lg) from the twiddle table (a reduced modulo 2^lg)
template <typename Rl, bool INV>
__device__ __forceinline__ cpx<Rl> tw_pow(const TwTab<Rl>& tw, unsigned a, int lg) {
    return twiddle<Rl, INV>(tw, (a & ((1u << lg) - 1)) << (TW_LOG_MMAX - lg));
}

// ------------------------------------------------------------------ real transform pair
// to_time! of a length-2Mc real signal from its spectrum X[n] = load(n), n < Nw (zero up to
// n = Mc): C2R pre-twiddle Z[n] = (X[n] + conj X[Mc-n]) + i W^-n (X[n] - conj X[Mc-n]) and
// an Mc-point inverse transform. On return tb holds this CTA's block of sample pairs
// m = rank Mbc + n1 (unscaled). load is called once for each own bin.
template <typename Rl, int R, typename LoadF>
__device__ __noinline__ void dist_c2r(DWs<Rl>& d, int Mc, int Nw, LoadF&& load) {
    const int p = d.rank, T = LUNA_BLOCK, tid = threadIdx.x;
    const int Mbc = Mc / R;
    const int lgM = ilog2i((unsigned)Mc), lgR = ilog2c<R>();
    // DUnr<R>::v own bins per thread and round: their loads are independent and issued together
    for (int j0 = tid; p + R * j0 <= Mc; j0 += DUnr<R>::v * T) {
        cpx<double> X[DUnr<R>::v];
#pragma unroll
        for (int u = 0; u < DUnr<R>::v; ++u) {
            const int n = p + R * (j0 + u * T);
            X[u] = (n < Nw) ? load(n) : mk<double>(0, 0);
        }
#pragma unroll
        for (int u = 0; u < DUnr<R>::v; ++u) {
            const int j = j0 + u * T;
            if (p + R * j <= Mc) d.stg[Swz<Rl>::f(j)] = cvt<Rl>(X[u]);
        }
    }
    dsync();
    const int po = (R - p) % R;
    const cpx<Rl>* so = drem(d.stg, po);
    // remote loads of DUnr<R>::v elements are issued before any is used (latency of the cluster)
    for (int k0 = tid; k0 < Mbc; k0 += DUnr<R>::v * T) {
        cpx<Rl> xm[DUnr<R>::v];
#pragma unroll
        for (int u = 0; u < DUnr<R>::v; ++u) {
            const int k = k0 + u * T;
            const int nm = Mc - (R * k + p);  // the partner bin, owned by CTA po
            xm[u] = (k < Mbc) ? so[Swz<Rl>::f((nm - po) / R)] : mk<Rl>(0, 0);
        }
#pragma unroll
        for (int u = 0; u < DUnr<R>::v; ++u) {
            const int k = k0 + u * T;
            if (k >= Mbc) continue;
            const int n = R * k + p;
            cpx<double> Xk = cvt<double>(d.stg[Swz<Rl>::f(k)]);
            cpx<double> Xm = cvt<double>(xm[u]);
            if (n == 0) {  // imaginary parts of DC and Nyquist do not enter a real transform
                Xk.y = 0;
                Xm.y = 0;
            }
            const cpx<double> Wi = half_twiddle<Rl, true>(d.tw, n, Mc);
            const cpx<double> Z = (Xk + conj(Xm)) + mul_mi<double, true>(Wi * (Xk - conj(Xm)));
            d.fb[Swz<Rl>::f(k)] = cvt<Rl>(Z);
        }
    }
    __syncthreads();
    sub_fft_any<Rl, true>(d.fb, Mbc, d.tw);
    if (p) {
        for (int n1 = tid; n1 < Mbc; n1 += T) {
            const int pos = Swz<Rl>::f(n1);
            d.fb[pos] = d.fb[pos] * tw_pow<Rl, true>(d.tw, (unsigned)(p * n1), lgM);
        }
    }
    dsync();
    if constexpr (R == 8 || R == 16) {
        // join, transposed: this CTA takes the n1 of its slice [p S, (p + 1) S), S = Mbc/R,
        // gathers B_r[n1] from every CTA, forms x[n1 + Mbc q] = sum_r W_R^{-r q} B_r[n1] for
        // every q with one in-register DFT and stores each into CTA q's block. Each CTA reads
        // Mbc values instead of R Mbc; the stores are visible after the closing barrier.
        const int S = Mbc / R, n1b = p * S;
        for (int j = tid; j < S; j += T) {
            const int pos = Swz<Rl>::f(n1b + j);
            cpx<Rl> v[R];
#pragma unroll
            for (int i = 0; i < R; ++i) v[i] = drem(d.fb, bitrev<R>(i))[pos];
            dft_br<Rl, true, R>(v);
#pragma unroll
            for (int q = 0; q < R; ++q) drem(d.tb, q)[pos] = v[q];
        }
        dsync();
    } else {
    // join: x[n1 + Mbc q] = sum_r W_R^{-r q} B_r[n1], q = this CTA
    const cpx<Rl>* fr[R];
    cpx<Rl> wq[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        fr[r] = drem(d.fb, r);
        wq[r] = tw_pow<Rl, true>(d.tw, (unsigned)(r * p), lgR);
    }
    for (int n0 = tid; n0 < Mbc; n0 += DUnr<R>::v * T) {
        cpx<Rl> v[DUnr<R>::v][R];
#pragma unroll
        for (int u = 0; u < DUnr<R>::v; ++u) {
            const int pos = Swz<Rl>::f(min(n0 + u * T, Mbc - 1));
#pragma unroll
            for (int r = 0; r < R; ++r) v[u][r] = fr[r][pos];
        }
#pragma unroll
        for (int u = 0; u < DUnr<R>::v; ++u) {
            if (n0 + u * T >= Mbc) continue;
            cpx<Rl> acc = v[u][0];
#pragma unroll
            for (int r = 1; r < R; ++r) acc = acc + v[u][r] * wq[r];
            d.tb[Swz<Rl>::f(n0 + u * T)] = acc;
        }
    }
    __syncthreads();
    }
}

// to_freq! of the sample pairs in tb (every CTA's block): radix-R step, Mbc-point forward
// sub-transform of this CTA's sub-sequence, R2C split
// X[k] = 1/2 (Z[k] + conj Z[Mc-k]) - i/2 W^k (Z[k] - conj Z[Mc-k]) and store(k, X) for the
// own bins k < Nw. Opens with a cluster barrier (every block complete, every remote read of
// the previous phase done).
template <typename Rl, int R, typename StoreF>
__device__ __noinline__ void dist_r2c(DWs<Rl>& d, int Mc, int Nw, StoreF&& store) {
    const int p = d.rank, T = LUNA_BLOCK, tid = threadIdx.x;
    const int Mbc = Mc / R;
    const int lgM = ilog2i((unsigned)Mc), lgR = ilog2c<R>();
    dsync();
    if constexpr (R == 8 || R == 16) {
        // radix-R step, transposed: this CTA takes the n1 of its slice, gathers every CTA's
        // block at n1, forms y_r = W_M^{r n1} sum_q W_R^{r q} x[n1 + Mbc q] for every r with
        // one in-register DFT and stores each into CTA r's sub-transform buffer
        const int S = Mbc / R, n1b = p * S;
        for (int j = tid; j < S; j += T) {
            const int n1 = n1b + j;
            const int pos = Swz<Rl>::f(n1);
            cpx<Rl> v[R];
#pragma unroll
            for (int i = 0; i < R; ++i) v[i] = drem(d.tb, bitrev<R>(i))[pos];
            dft_br<Rl, false, R>(v);
            drem(d.fb, 0)[pos] = v[0];
#pragma unroll
            for (int r = 1; r < R; ++r) drem(d.fb, r)[pos] = v[r] * tw_pow<Rl, false>(d.tw, (unsigned)(r * n1), lgM);
        }
        dsync();
    } else {
    const cpx<Rl>* tr[R];
    cpx<Rl> wq[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
        tr[q] = drem(d.tb, q);
        wq[q] = tw_pow<Rl, false>(d.tw, (unsigned)(p * q), lgR);
    }
    for (int n0 = tid; n0 < Mbc; n0 += DUnr<R>::v * T) {
        cpx<Rl> v[DUnr<R>::v][R];
#pragma unroll
        for (int u = 0; u < DUnr<R>::v; ++u) {
            const int pos = Swz<Rl>::f(min(n0 + u * T, Mbc - 1));
#pragma unroll
            for (int q = 0; q < R; ++q) v[u][q] = tr[q][pos];
        }
#pragma unroll
        for (int u = 0; u < DUnr<R>::v; ++u) {
            const int n1 = n0 + u * T;
            if (n1 >= Mbc) continue;
            cpx<Rl> acc = v[u][0];
#pragma unroll
            for (int q = 1; q < R; ++q) acc = acc + v[u][q] * wq[q];
            if (p) acc = acc * tw_pow<Rl, false>(d.tw, (unsigned)(p * n1), lgM);
            d.fb[Swz<Rl>::f(n1)] = acc;
        }
    }
    __syncthreads();
    }
    sub_fft_any<Rl, false>(d.fb, Mbc, d.tw);
    dsync();
    const int po = (R - p) % R;
    const cpx<Rl>* fo = drem(d.fb, po);
    for (int j0 = tid; p + R * j0 < Nw; j0 += DUnr<R>::v * T) {
      cpx<Rl> zm[DUnr<R>::v];
#pragma unroll
      for (int u = 0; u < DUnr<R>::v; ++u) {
          const int k = p + R * (j0 + u * T);
          zm[u] = (k < Nw) ? fo[Swz<Rl>::f(((Mc - k) & (Mc - 1)) / R)] : mk<Rl>(0, 0);
      }
#pragma unroll
      for (int u = 0; u < DUnr<R>::v; ++u) {
        const int k = p + R * (j0 + u * T);
        if (k >= Nw) continue;
        const int kk = k & (Mc - 1);
        const cpx<double> Zk = cvt<double>(d.fb[Swz<Rl>::f(kk / R)]);
        const cpx<double> Zm = cvt<double>(zm[u]);
        cpx<double> X;
        if (k == 0) X = mk<double>(Zk.x + Zk.y, 0.0);
        else if (k == Mc) X = mk<double>(Zk.x - Zk.y, 0.0);
        else {
            const cpx<double> Wk = half_twiddle<Rl, false>(d.tw, k, Mc);
            X = scale(0.5, Zk + conj(Zm)) + scale(0.5, mul_mi<double, false>(Wk * (Zk - conj(Zm))));
        }
        store(k, X);
      }
    }
    __syncthreads();
}

// ------------------------------------------------------------------ Raman convolution
// The 2M-point transform of z[m] = (E[2m]^2, E[2m+1]^2) (m < M, zero above) on 2R
// sub-transforms of Mb points, its real-transform split, the response product and the
// inverse split (as raman_conv), then the inverse sub-transforms; rb0/rb1 end holding
// B_p[n1] = W_2M^{-p n1} IFFT_Mb(Y_p)[n1] for this CTA's pair of sub-transforms. Needs
// every CTA's field block (call after a cluster barrier).
template <typename Rl, int R>
__device__ __noinline__ void dist_raman_fwd(const LunaResp& rr, DWs<Rl>& d, int M, double sc) {
    const int c = d.rank, T = LUNA_BLOCK, tid = threadIdx.x;
    const int Mb = M / R, Mr = 2 * M;
    const int lgMr = ilog2i((unsigned)Mr), lg2R = ilog2c<R>() + 1;
    const int pa = (c == 0) ? 0 : c, pb = (c == 0) ? R : 2 * R - c;
    const Rl s = (Rl)sc;
    if constexpr (R == 8) {
        // the radix-2R step, transposed: this CTA takes the n1 of its slice, squares every
        // CTA's field pair at n1, forms X_f = sum_q W_2R^{f q} z[n1 + Mb q] for all 2R
        // sub-transforms f with one in-register DFT (z is zero for q >= R) and stores
        // X_f W_2M^{f n1} into the buffer of the CTA that owns f (f = c and 2R - c of CTA c,
        // 0 and R of CTA 0)
        constexpr int R2 = 2 * R;
        const int S = Mb / R, n1b = c * S;
        for (int j = tid; j < S; j += T) {
            const int n1 = n1b + j;
            const int pos = Swz<Rl>::f(n1);
            cpx<Rl> v[R2];
#pragma unroll
            for (int i = 0; i < R2; ++i) {
                const int q = bitrev<R2>(i);
                if (q < R) {
                    const cpx<Rl> e = drem(d.tb, q)[pos];
                    const Rl e0 = e.x * s, e1 = e.y * s;
                    v[i] = mk<Rl>(e0 * e0, e1 * e1);
                } else {
                    v[i] = mk<Rl>(0, 0);
                }
            }
            dft_br<Rl, false, R2>(v);
            drem(d.rb0, 0)[pos] = v[0];
            drem(d.rb1, 0)[pos] = v[R] * tw_pow<Rl, false>(d.tw, (unsigned)(R * n1), lgMr);
#pragma unroll
            for (int cc = 1; cc < R; ++cc) {
                drem(d.rb0, cc)[pos] = v[cc] * tw_pow<Rl, false>(d.tw, (unsigned)(cc * n1), lgMr);
                drem(d.rb1, cc)[pos] = v[R2 - cc] * tw_pow<Rl, false>(d.tw, (unsigned)((R2 - cc) * n1), lgMr);
            }
        }
        dsync();
    } else if constexpr (R == 16) {
        // the same transposed step with the 2R-point DFT as two R-point ones (a 2R-point
        // one does not fit in registers): z is zero for q >= R, so
        // X_{2g+e} = sum_{q<R} W_R^{g q} (W_2R^{e q} z_q), e = 0, 1; each half gathers the
        // squares again instead of holding them
        const int S = Mb / R, n1b = c * S;
        for (int j = tid; j < S; j += T) {
            const int n1 = n1b + j;
            const int pos = Swz<Rl>::f(n1);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                cpx<Rl> v[R];
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    const int q = bitrev<R>(i);
                    const cpx<Rl> ev = drem(d.tb, q)[pos];
                    const Rl e0 = ev.x * s, e1 = ev.y * s;
                    v[i] = mk<Rl>(e0 * e0, e1 * e1);
                    if (e && q) v[i] = v[i] * tw_pow<Rl, false>(d.tw, (unsigned)q, lg2R);
                }
                dft_br<Rl, false, R>(v);
#pragma unroll
                for (int g = 0; g < R; ++g) {
                    const int f = 2 * g + e;  // sub-transform f: rb0 of CTA f (f < R), rb1 of CTA 2R - f
                    if (f == 0) drem(d.rb0, 0)[pos] = v[g];
                    else if (f < R) drem(d.rb0, f)[pos] = v[g] * tw_pow<Rl, false>(d.tw, (unsigned)(f * n1), lgMr);
                    else drem(d.rb1, f == R ? 0 : 2 * R - f)[pos] = v[g] * tw_pow<Rl, false>(d.tw, (unsigned)(f * n1), lgMr);
                }
            }
        }
        dsync();
    } else {
    const cpx<Rl>* tr[R];
    cpx<Rl> wa[R], wb[R];
#pragma unroll
    for (int q = 0; q < R; ++q) {
        tr[q] = drem(d.tb, q);
        wa[q] = tw_pow<Rl, false>(d.tw, (unsigned)(pa * q), lg2R);
        wb[q] = tw_pow<Rl, false>(d.tw, (unsigned)(pb * q), lg2R);
    }
    for (int n0 = tid; n0 < Mb; n0 += DUnr<R>::v * T) {
      cpx<Rl> ev[DUnr<R>::v][R];
#pragma unroll
      for (int u = 0; u < DUnr<R>::v; ++u) {
          const int pos = Swz<Rl>::f(min(n0 + u * T, Mb - 1));
#pragma unroll
          for (int q = 0; q < R; ++q) ev[u][q] = tr[q][pos];
      }
#pragma unroll
      for (int u = 0; u < DUnr<R>::v; ++u) {
        const int n1 = n0 + u * T;
        if (n1 >= Mb) continue;
        const int pos = Swz<Rl>::f(n1);
        cpx<Rl> z[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const cpx<Rl> e = ev[u][q];
            const Rl e0 = e.x * s, e1 = e.y * s;
            z[q] = mk<Rl>(e0 * e0, e1 * e1);
        }
        cpx<Rl> a = z[0], b = z[0];
#pragma unroll
        for (int q = 1; q < R; ++q) {
            a = a + z[q] * wa[q];
            b = b + z[q] * wb[q];
        }
        if (pa) a = a * tw_pow<Rl, false>(d.tw, (unsigned)(pa * n1), lgMr);
        b = b * tw_pow<Rl, false>(d.tw, (unsigned)(pb * n1), lgMr);
        d.rb0[pos] = a;
        d.rb1[pos] = b;
      }
    }
    __syncthreads();
    }
    sub_fft2<Rl, false, 8>(d.rb0, d.rb1, Mb, d.tw);
    // pairs (f, Mr - f) with f = 2R k + p; Zk/Zm are entries of the complex transform
    const cpx<Rl>* H = reinterpret_cast<const cpx<Rl>*>(rr.H);
    auto pair = [&](int f, cpx<Rl>* bk, int ik, cpx<Rl>* bm, int im) {
        const int fm = (Mr - f) & (Mr - 1);
        const cpx<double> Zk = cvt<double>(bk[Swz<Rl>::f(ik)]);
        const cpx<double> Zm = cvt<double>(bm[Swz<Rl>::f(im)]);
        const cpx<double> Wk = half_twiddle<Rl, false>(d.tw, f, Mr);
        cpx<double> Xk, Xm;
        if (f == 0) {
            Xk = mk<double>(Zk.x + Zk.y, 0.0);
            Xm = mk<double>(Zk.x - Zk.y, 0.0);
        } else {
            Xk = scale(0.5, Zk + conj(Zm)) + scale(0.5, mul_mi<double, false>(Wk * (Zk - conj(Zm))));
            const cpx<double> Wm = scale(-1.0, conj(Wk));
            Xm = scale(0.5, Zm + conj(Zk)) + scale(0.5, mul_mi<double, false>(Wm * (Zm - conj(Zk))));
        }
        const cpx<double> Yk = Xk * cvt<double>(ldg(H + f));
        const cpx<double> Ym = Xm * cvt<double>(ldg(H + (Mr - f)));
        const cpx<double> Wi = conj(Wk);
        const cpx<double> Zk2 = (Yk + conj(Ym)) + mul_mi<double, true>(Wi * (Yk - conj(Ym)));
        bk[Swz<Rl>::f(ik)] = cvt<Rl>(Zk2);
        if (f != 0 && fm != f) {
            const cpx<double> Wmi = scale(-1.0, Wk);
            const cpx<double> Zm2 = (Ym + conj(Yk)) + mul_mi<double, true>(Wmi * (Ym - conj(Yk)));
            bm[Swz<Rl>::f(im)] = cvt<Rl>(Zm2);
        }
    };
    if (c == 0) {
        // sub-transform 0: f = 2R k pairs with index Mb - k (k = 0 and k = Mb/2 alone);
        // sub-transform R: f = 2R k + R pairs with index Mb - 1 - k
        for (int k = tid; k <= Mb / 2; k += T) pair(2 * R * k, d.rb0, k, d.rb0, (Mb - k) & (Mb - 1));
        for (int k = tid; k < Mb / 2; k += T) pair(2 * R * k + R, d.rb1, k, d.rb1, Mb - 1 - k);
    } else {
        // f = 2R k + c in rb0 pairs with 2R (Mb - 1 - k) + (2R - c) in rb1
        for (int k = tid; k < Mb; k += T) pair(2 * R * k + c, d.rb0, k, d.rb1, Mb - 1 - k);
    }
    __syncthreads();
    sub_fft2<Rl, true, 8>(d.rb0, d.rb1, Mb, d.tw);
    for (int n1 = tid; n1 < Mb; n1 += T) {
        const int pos = Swz<Rl>::f(n1);
        if (pa) d.rb0[pos] = d.rb0[pos] * tw_pow<Rl, true>(d.tw, (unsigned)(pa * n1), lgMr);
        d.rb1[pos] = d.rb1[pos] * tw_pow<Rl, true>(d.tw, (unsigned)(pb * n1), lgMr);
    }
    __syncthreads();
}

// Raman polarisation pair of this CTA's block at n1 from every CTA's B_p (after a barrier
// that follows dist_raman_fwd in every CTA): P[n1 + Mb q] = sum_p W_2R^{-p q} B_p[n1].
template <typename Rl, int R>
struct RamanOut {
    const cpx<Rl>* b0[R];
    const cpx<Rl>* b1[R];
    cpx<Rl> w0[R], w1[R];
    __device__ void init(DWs<Rl>& d) {
        const int q = d.rank, lg2R = ilog2c<R>() + 1;
#pragma unroll
        for (int c = 0; c < R; ++c) {
            b0[c] = drem(d.rb0, c);
            b1[c] = drem(d.rb1, c);
            const int pa = (c == 0) ? 0 : c, pb = (c == 0) ? R : 2 * R - c;
            w0[c] = tw_pow<Rl, true>(d.tw, (unsigned)(pa * q), lg2R);
            w1[c] = tw_pow<Rl, true>(d.tw, (unsigned)(pb * q), lg2R);
        }
    }
    // P for the pairs n1 = tid + k T of this CTA's block into out[Swz(n1)] (remote loads of
    // two pairs in flight together)
    __device__ void block(cpx<Rl>* out, int Mb) const {
        constexpr int U = DUnr<R>::raman;
        for (int n0 = threadIdx.x; n0 < Mb; n0 += U * LUNA_BLOCK) {
            cpx<Rl> v0[U][R], v1[U][R];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int pos = Swz<Rl>::f(min(n0 + u * LUNA_BLOCK, Mb - 1));
#pragma unroll
                for (int c = 0; c < R; ++c) {
                    v0[u][c] = b0[c][pos];
                    v1[u][c] = b1[c][pos];
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int n1 = n0 + u * LUNA_BLOCK;
                if (n1 >= Mb) continue;
                cpx<Rl> acc = v0[u][0] + v1[u][0] * w1[0];
#pragma unroll
                for (int c = 1; c < R; ++c) acc = acc + v0[u][c] * w0[c] + v1[u][c] * w1[c];
                out[Swz<Rl>::f(n1)] = acc;
            }
        }
    }
    __device__ __forceinline__ cpx<Rl> at(int pos) const {
        cpx<Rl> v0[R], v1[R];
#pragma unroll
        for (int c = 0; c < R; ++c) {
            v0[c] = b0[c][pos];
            v1[c] = b1[c][pos];
        }
        cpx<Rl> acc = v0[0] + v1[0] * w1[0];
#pragma unroll
        for (int c = 1; c < R; ++c) acc = acc + v0[c] * w0[c] + v1[c] * w1[c];
        return acc;
    }
};

// RamanOut::block transposed for clusters of 8 and 16: this CTA takes the n1 of its slice
// [r S, (r + 1) S), S = Mb/R, gathers the 2R sub-transform values B_p[n1] (two per CTA),
// forms P[n1 + Mb q] = sum_p W_2R^{-p q} B_p[n1] for every q with one in-register DFT and
// stores each into CTA q's out. Each CTA reads 2 Mb values instead of 2 R Mb; the stores
// are visible to CTA q after the next cluster barrier.
// For R = 16 the 2R-point DFT runs as two R-point ones over p = g + R e:
// P_{2h} = IDFT_R(B_g + B_{g+R})[h] and P_{2h+1} = IDFT_R((B_g - B_{g+R}) W_2R^{-g})[h],
// h < R/2 (only q < R is wanted); each half gathers the 2R values again.
template <typename Rl, int R>
__device__ __forceinline__ void raman_out_scatter(DWs<Rl>& d, cpx<Rl>* out, int Mb) {
    constexpr int R2 = 2 * R;
    const int S = Mb / R, n1b = d.rank * S;
    if constexpr (R == 16) {
        constexpr int lg2R = ilog2c<R2>();
        for (int j = threadIdx.x; j < S; j += LUNA_BLOCK) {
            const int pos = Swz<Rl>::f(n1b + j);
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                cpx<Rl> v[R];
#pragma unroll
                for (int i = 0; i < R; ++i) {
                    const int g = bitrev<R>(i);
                    const cpx<Rl> a = drem(d.rb0, g)[pos];                   // B_g
                    const cpx<Rl> b = drem(d.rb1, g == 0 ? 0 : R - g)[pos];  // B_{g+R}
                    v[i] = e ? (g ? (a - b) * tw_pow<Rl, true>(d.tw, (unsigned)g, lg2R) : a - b) : a + b;
                }
                dft_br<Rl, true, R>(v);
#pragma unroll
                for (int h = 0; h < R / 2; ++h) drem(out, 2 * h + e)[pos] = v[h];
            }
        }
        return;
    }
    for (int j = threadIdx.x; j < S; j += LUNA_BLOCK) {
        const int pos = Swz<Rl>::f(n1b + j);
        cpx<Rl> x[R2];
#pragma unroll
        for (int c = 0; c < R; ++c) {
            x[c] = drem(d.rb0, c)[pos];
            x[c == 0 ? R : R2 - c] = drem(d.rb1, c)[pos];
        }
        cpx<Rl> v[R2];
#pragma unroll
        for (int i = 0; i < R2; ++i) v[i] = x[bitrev<R2>(i)];
        dft_br<Rl, true, R2>(v);
#pragma unroll
        for (int q = 0; q < R; ++q) drem(out, q)[pos] = v[q];
    }
}

// ------------------------------------------------------------------ plasma
// The rate-function parameters in registers (ppt_rate<float> / adk_rate<float> with the
// same arithmetic), read once per call instead of once per sample.
struct RateF {
    int ppt, n;
    float xmin, xmax, thr, a, b, pw, lpre;
    const float *sx, *sy, *sD;
    __device__ void init(const LunaResp& r) {
        ppt = r.kind == LUNA_RESP_PLASMA_PPT;
        n = r.sn;
        xmin = (float)r.Emin;
        xmax = (float)r.Emax;
        sx = r.sxf;
        sy = r.syf;
        sD = r.sDf;
        thr = (float)r.adk_thr;
        a = (float)r.adk_a;
        b = (float)r.adk_b;
        pw = (float)r.adk_pw;
        lpre = logf((float)r.adk_pre);
    }
    __device__ __forceinline__ float operator()(float aE, int* flag) const {
        if (ppt) {
            if (aE < xmin) return 0.0f;
            if (aE > xmax) {
                atomicOr(flag, 1 << ST_FIELD_ABOVE_EMAX);
                return 0.0f;
            }
            int i1 = (int)ceilf((aE - xmin) / (xmax - xmin) * (float)(n - 1)) + 1;
            i1 = max(2, min(n, i1));
            const int i = i1 - 1;
            const float xi = __ldg(sx + i), xm = __ldg(sx + i - 1);
            const float yi = __ldg(sy + i), ym = __ldg(sy + i - 1);
            const float Di = __ldg(sD + i), Dm = __ldg(sD + i - 1);
            const float t = (aE - xm) / (xi - xm);
            const float v = ym + Dm * t + (3.0f * (yi - ym) - 2.0f * Dm - Di) * (t * t)
                            + (2.0f * (ym - yi) + Dm + Di) * (t * t * t);
            return expf(v);
        }
        if (aE < thr || aE == 0.0f) return 0.0f;
        return expf(pw * logf(a / aE) - b / aE + lpre);
    }
};

// PlasmaScalar! (Nonlinear.jl:121-133) with Kerr, Raman and the time window on this CTA's
// block, every thread holding NS consecutive samples: three cumulative trapezoids written
// as prefix sums (FP64), each one block scan, with the carries into the block (the totals
// of the CTAs before it) and the integrands' first samples exchanged through the cluster.
// Mixed precision: rates, ionisation fractions (1 - exp(-x) as -expm1(-x)) and the
// ionisation-loss current are FP32 per sample (kept in shared memory at [s*T + tid]
// between the passes), the running integrals FP64. FP64: every quantity FP64.
template <typename Rl, int NS, int R>
__device__ __noinline__ void dist_plasma(const LunaInst& I, DWs<Rl>& d, int M, double sc, int ip, int ir, double kc,
                                         double rc) {
    const int q = d.rank, T = LUNA_BLOCK, tid = threadIdx.x;
    const int Mb = M / R;
    const int mbase = q * Mb;
    const LunaResp& r = I.resp[ip];
    const double dt = r.dt, er = r.eratio, preion = r.preion, coef = r.coef;
    const float ipf = (float)r.ionpot;
    const int pr0 = tid * (NS / 2);
    // per-sample rates and ionisation fractions in the solver's precision: FP32 in mixed
    // precision, FP64 (the arithmetic of the single-CTA FP64 plasma scan) otherwise
    constexpr bool F64 = sizeof(Rl) == 8;
    Rl* rrb = reinterpret_cast<Rl*>(d.stg);  // rates (the staged spectrum is dead)
    Rl* frb = reinterpret_cast<Rl*>(d.fb);   // ionisation fractions
    Rl ev[NS];  // stored field samples; E = ev * sc
#pragma unroll
    for (int h = 0; h < NS / 2; ++h) {
        const cpx<Rl> e = d.tb[Swz<Rl>::f(pr0 + h)];
        ev[2 * h] = e.x;
        ev[2 * h + 1] = e.y;
    }
    auto E = [&](int s) -> double { return (double)ev[s] * sc; };
    // pass A: rates; exclusive scan of the thread sums and the block total
    double racc = 0;
    Rl r0 = 0;
    if constexpr (F64) {
        const bool ppt = r.kind == LUNA_RESP_PLASMA_PPT;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double aE = fabs(E(s));
            const double rv = ppt ? ppt_rate<double>(r, aE, d.flag) : adk_rate<double>(r, aE);
            rrb[s * T + tid] = rv;
            racc += rv;
            if (s == 0) r0 = rv;
        }
    } else {
        RateF rf;
        rf.init(r);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const float rv = rf((float)fabs(E(s)), d.flag);
            rrb[s * T + tid] = rv;
            racc += (double)rv;
            if (s == 0) r0 = rv;
        }
    }
    double tot;
    const double xr = block_exscan(racc, d.tot, tot);
    if (tid == 0) {
        d.xs[0] = tot;
        d.xs[1] = r0;
    }
    dsync();  // totals published; Raman sub-transforms ready; field blocks no longer read
    if (ir >= 0) {
        // the Raman polarisation of this block into tb (the field now lives in ev); with the
        // transposed form other CTAs write it, visible after the next barriers below
        if constexpr (R == 8 || R == 16) {
            raman_out_scatter<Rl, R>(d, d.tb, Mb);
        } else {
            RamanOut<Rl, R> ro;
            ro.init(d);
            ro.block(d.tb, Mb);
        }
    }
    double c1 = 0;
    for (int j = 0; j < q; ++j) c1 += drem(d.xs, j)[0];
    const double y0r = drem(d.xs, 0)[1];
    // pass B: ionisation fractions, phase-integrand sums
    double ph_acc = 0, ph_first = 0;
    {
        double S = c1 + xr;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double rr = rrb[s * T + tid];
            S += rr;
            Rl fr;
            if constexpr (F64) {
                const double f = dt * (S - 0.5 * (y0r + rr));
                fr = preion + 1.0 - ((f == 0.0) ? 1.0 : exp(-f));
            } else {
                const float fx = (float)(dt * (S - 0.5 * (y0r + rr)));
                fr = (float)(preion - (double)expm1f(-fx));
            }
            frb[s * T + tid] = fr;
            const double ph = (double)fr * er * E(s);
            ph_acc += ph;
            if (s == 0) ph_first = ph;
        }
    }
    const double xp = block_exscan(ph_acc, d.tot + LUNA_WARPS, tot);
    if (tid == 0) {
        d.xs[2] = tot;
        d.xs[3] = ph_first;
    }
    dsync();
    double c2 = 0;
    for (int j = 0; j < q; ++j) c2 += drem(d.xs, j)[2];
    const double y0p = drem(d.xs, 0)[3];
    // the current density of sample s, advancing the running phase integral Tv
    auto current = [&](int s, double& Tv) -> double {
        const Rl rr = rrb[s * T + tid], fr = frb[s * T + tid];
        const double ph = (double)fr * er * E(s);
        Tv += ph;
        double ion;
        if constexpr (F64) {
            const double Es = E(s);
            ion = (fabs(Es) > 0) ? r.ionpot * rr * (1.0 - fr) / Es : 0.0;
        } else {
            const float Ef = (float)E(s);
            ion = (double)((Ef != 0.0f) ? ipf * rr * (1.0f - fr) / Ef : 0.0f);
        }
        return dt * (Tv - 0.5 * (y0p + ph)) + ion;
    };
    double J_acc = 0, J_first = 0;
    {
        double Tv = c2 + xp;
#pragma unroll
        for (int s = 0; s < NS; ++s) {
            const double J = current(s, Tv);
            J_acc += J;
            if (s == 0) J_first = J;
        }
    }
    const double xj = block_exscan(J_acc, d.tot + 2 * LUNA_WARPS, tot);
    if (tid == 0) {
        d.xs[4] = tot;
        d.xs[5] = J_first;
    }
    dsync();
    double c3 = 0;
    for (int j = 0; j < q; ++j) c3 += drem(d.xs, j)[4];
    const double y0J = drem(d.xs, 0)[5];
    // polarisation, Kerr and Raman terms, time window
    cpx<Rl> rman[NS / 2];
    if (ir >= 0) {
        __syncthreads();  // the Raman block written above by other threads
#pragma unroll
        for (int h = 0; h < NS / 2; ++h) rman[h] = d.tb[Swz<Rl>::f(pr0 + h)];
    }
    double Tv = c2 + xp, U = c3 + xj;
#pragma unroll
    for (int h = 0; h < NS / 2; ++h) {
        double P[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            const int s = 2 * h + c;
            const double J = current(s, Tv);
            U += J;
            const double Es = E(s);
            P[c] = kc * (Es * Es * Es) + coef * (dt * (U - 0.5 * (y0J + J)));
            if (ir >= 0) P[c] += rc * Es * (double)(c ? rman[h].y : rman[h].x);
        }
        const double2 tw = __ldg(reinterpret_cast<const double2*>(I.towin) + mbase + pr0 + h);
        d.tb[Swz<Rl>::f(pr0 + h)] = mk<Rl>((Rl)(P[0] * tw.x), (Rl)(P[1] * tw.y));
    }
    __syncthreads();
}

// ------------------------------------------------------------------ responses
// Et_to_Pt! and the time window on this CTA's block (PlasmaScalar!, Nonlinear.jl:121-133,
// as running trapezoids written as prefix sums; the carries into the block are the block
// totals of the CTAs before it, exchanged through the cluster).
template <typename Rl, int R>
__device__ __noinline__ void dist_pointwise(const LunaInst& I, DWs<Rl>& d, int M, double sc) {
    const int q = d.rank, T = LUNA_BLOCK, tid = threadIdx.x;
    const int Mb = M / R;
    const int mbase = q * Mb;
    int ip = -1, ir = -1;
    for (int i = 0; i < I.nresp; ++i) {
        if (I.resp[i].kind == LUNA_RESP_PLASMA_PPT || I.resp[i].kind == LUNA_RESP_PLASMA_ADK) ip = i;
        if (I.resp[i].kind == LUNA_RESP_RAMAN) ir = i;
    }
    double kc = 0, rc = 0;  // Kerr and Raman coefficients
    for (int i = 0; i < I.nresp; ++i) {
        if (I.resp[i].kind == LUNA_RESP_KERR_FIELD) kc += I.resp[i].coef;
        if (i == ir) rc = I.resp[i].coef;
    }
    if (ip < 0 && ir < 0) {
        for (int n1 = tid; n1 < Mb; n1 += T) {
            const int pos = Swz<Rl>::f(n1);
            const cpx<Rl> e = d.tb[pos];
            const double E0 = (double)e.x * sc, E1 = (double)e.y * sc;
            const double2 tw = __ldg(reinterpret_cast<const double2*>(I.towin) + mbase + n1);
            d.tb[pos] = mk<Rl>((Rl)(kc * (E0 * E0 * E0) * tw.x), (Rl)(kc * (E1 * E1 * E1) * tw.y));
        }
        __syncthreads();
        return;
    }
    dsync();  // every field block complete; every read of the sub-transforms done
    if (ir >= 0) dist_raman_fwd<Rl, R>(I.resp[ir], d, M, sc);
    if (ip < 0) {
        dsync();  // every CTA's Raman sub-transforms ready; every read of the field blocks done
        // the sub-transform buffer is free after the barrier above
        if constexpr (R == 8 || R == 16) {
            raman_out_scatter<Rl, R>(d, d.fb, Mb);
            dsync();  // every CTA's stores into this block
        } else {
            RamanOut<Rl, R> ro;
            ro.init(d);
            ro.block(d.fb, Mb);
            __syncthreads();
        }
        for (int n1 = tid; n1 < Mb; n1 += T) {
            const int pos = Swz<Rl>::f(n1);
            const cpx<Rl> e = d.tb[pos];
            const cpx<Rl> pr = d.fb[pos];
            const double E0 = (double)e.x * sc, E1 = (double)e.y * sc;
            const double P0 = kc * (E0 * E0 * E0) + rc * E0 * (double)pr.x;
            const double P1 = kc * (E1 * E1 * E1) + rc * E1 * (double)pr.y;
            const double2 tw = __ldg(reinterpret_cast<const double2*>(I.towin) + mbase + n1);
            d.tb[pos] = mk<Rl>((Rl)(P0 * tw.x), (Rl)(P1 * tw.y));
        }
        __syncthreads();
        return;
    }
    switch (2 * Mb / T) {  // samples per thread
        case 4: dist_plasma<Rl, 4, R>(I, d, M, sc, ip, ir, kc, rc); break;
        case 8: dist_plasma<Rl, 8, R>(I, d, M, sc, ip, ir, kc, rc); break;
        default: dist_plasma<Rl, 16, R>(I, d, M, sc, ip, ir, kc, rc); break;
    }
}

// ------------------------------------------------------------------ the integrator
// solve_instance for a distributed instance; every CTA of the cluster runs it.
template <typename Rl, typename Kt, int R>
__device__ __noinline__ void solve_instance_dist(LunaInst& I, DWs<Rl>& d, Ctl& c) {
    const int p = d.rank, T = LUNA_BLOCK, tid = threadIdx.x;
    const int Nw = I.Nw, M = I.No / 2, Mcoarse = I.N / 2;
    const bool writer = (p == 0);
    const cpx<double>* L = reinterpret_cast<const cpx<double>*>(I.linop);
    const cpx<double>* of = reinterpret_cast<const cpx<double>*>(I.outfac);
    void** k = c.k;
    if (tid == 0) {
        for (int j = 0; j < 7; ++j) k[j] = I.k[j];
        c.t = c.tn = I.z0;
        c.dt = c.dtn = I.dz0;
        c.err = c.errlast = 0;
        c.ok = 0;
        c.done = 0;
        c.status = 0;
        c.repeated = 0;
        c.steps = 0;
        *d.flag = 0;
    }
    cpx<double>* e1 = reinterpret_cast<cpx<double>*>(I.e1);
    double2* py = I.y;
    double2* pyn = I.yn;
    long long nrhs = 0;
    // the own bins n = p + R j
    auto own = [&](int t) { return p + R * t; };
    {
        const cpx<double>* y0 = reinterpret_cast<const cpx<double>*>(I.y0);
        cpx<double>* y = reinterpret_cast<cpx<double>*>(py);
        cpx<double>* yn = reinterpret_cast<cpx<double>*>(pyn);
        for (int t = tid; own(t) < Nw; t += T) {
            const int i = own(t);
            y[i] = y0[i];
            yn[i] = y0[i];
        }
    }
    __syncthreads();
    const double sc = I.in_scale;
    auto rhs_d = [&](auto&& load, auto&& store) {
        dist_c2r<Rl, R>(d, M, Nw, load);
        dist_pointwise<Rl, R>(I, d, M, sc);
        dist_r2c<Rl, R>(d, M, Nw, [&](int kb, cpx<double> X) { store(kb, X * ldg(of + kb)); });
    };
    {
        const cpx<double>* y = reinterpret_cast<const cpx<double>*>(py);
        void* k0 = k[0];
        rhs_d([&](int i) { return y[i]; }, [&](int i, cpx<double> v) { KT<Kt>::st(k0, i, v); });
        ++nrhs;
    }
    int saved = 0;
    bool swap_y = false;
    while (true) {
        __syncthreads();
        if (!(c.tn <= I.zmax) || c.done) break;
        if (swap_y) {
            double2* tmp = py;
            py = pyn;
            pyn = tmp;
        }
        const double dprop = c.tn - c.t;
        __syncthreads();
        if (tid == 0) {
            c.dt = c.dtn;
            c.t = c.tn;
        }
        __syncthreads();
        const double t0 = c.t, dt = c.dt;
        const cpx<double>* y = reinterpret_cast<const cpx<double>*>(py);
        for (int s = 0; s < 6; ++s) {
            const double zs = __dadd_rn(t0, __dmul_rn(c_nodes[s], dt));
            const double dd = __dsub_rn(zs, t0);
            if (s != 5) {
                for (int t0 = tid; own(t0) < Nw; t0 += DUnr<R>::v * T) {
                    cpx<double> Lv[DUnr<R>::v];
#pragma unroll
                    for (int u = 0; u < DUnr<R>::v; ++u) {
                        const int i = own(t0 + u * T);
                        Lv[u] = (i < Nw) ? ldg(L + i) : mk<double>(0, 0);
                    }
#pragma unroll
                    for (int u = 0; u < DUnr<R>::v; ++u) {
                        const int t = t0 + u * T, i = own(t);
                        if (i >= Nw) continue;
                        const cpx<Rl> f = expLd<Rl>(Lv[u], dd);
                        d.ef[Swz<Rl>::f(t)] = f;
                        if (s == 4) e1[i] = cvt<double>(f);
                    }
                }
            }
            __syncthreads();
            void* kout = k[s + 1];
            void* k1p = k[0];
            const double c0 = dt * c_B[s][0];
            const bool propk1 = (s == 0) && (dprop != 0.0);
            auto load = [&](int i) -> cpx<double> {
                cpx<double> k1 = KT<Kt>::ld(k1p, i);
                if (propk1) {
                    k1 = k1 * e1[i];
                    KT<Kt>::st(k1p, i, k1);
                }
                cpx<double> acc = y[i];
                acc = acc + scale(c0, k1);
                for (int j = 1; j <= s; ++j) {
                    const double bj = c_B[s][j];
                    if (bj != 0) acc = acc + scale(dt * bj, KT<Kt>::ld(k[j], i));
                }
                return cvt<double>(d.ef[Swz<Rl>::f((i - p) / R)]) * acc;
            };
            auto store = [&](int i, cpx<double> v) {
                KT<Kt>::st(kout, i, v * inv_fac<Rl>(d.ef[Swz<Rl>::f((i - p) / R)]));
            };
            rhs_d(load, store);
            ++nrhs;
        }
        // step! combine and this CTA's share of the weak-norm sums
        double sy = 0, syn = 0, se = 0;
        {
            cpx<double>* yn = reinterpret_cast<cpx<double>*>(pyn);
            double cb5[7], cer[7];
#pragma unroll
            for (int j = 0; j < 7; ++j) {
                cb5[j] = dt * c_b5[j];
                cer[j] = c_b5[j] - c_b4[j];
            }
            for (int t = tid; own(t) < Nw; t += T) {
                const int i = own(t);
                const cpx<double> yi = y[i];
                cpx<double> acc = yi;
                cpx<double> er = mk<double>(0, 0);
#pragma unroll
                for (int j = 0; j < 7; ++j) {
                    const cpx<double> kj = KT<Kt>::ld(k[j], i);
                    if (c_b5[j] != 0) acc = acc + scale(cb5[j], kj);
                    if (cer[j] != 0) er = er + scale(cer[j], scale(dt, kj));
                }
                yn[i] = acc;
                sy += abs2(yi);
                syn += abs2(acc);
                se += abs2(er);
            }
        }
        block_sum3(sy, syn, se, d.red);
        if (tid == 0) {
            d.xs[8] = sy;
            d.xs[9] = syn;
            d.xs[10] = se;
            d.xs[11] = (double)*d.flag;
        }
        dsync();
        if (tid == 0) {
            // every CTA sums the same partials in the same order: identical decisions
            double Sy = 0, Syn = 0, Se = 0;
            int fl = 0;
            for (int j = 0; j < R; ++j) {
                const double* x = drem(d.xs, j);
                Sy += x[8];
                Syn += x[9];
                Se += x[10];
                fl |= (int)x[11];
            }
            control_step(I, c, Sy, Syn, Se, fl, writer);
        }
        __syncthreads();
        if (c.done && c.status != 0) break;
        if (c.ok) {
            __syncthreads();
            if (tid == 0) {
                void* tmp = k[0];
                k[0] = k[6];
                k[6] = tmp;
            }
            __syncthreads();
            // prop!_maybe + stepfun window filter on yn (Luna.jl:366-372), on the coarse grid
            {
                cpx<double>* Yo = reinterpret_cast<cpx<double>*>(pyn);
                const double inv = 1.0 / (double)I.N;
                dist_c2r<Rl, R>(d, Mcoarse, Nw, [&](int i) -> cpx<double> {
                    return scale(__ldg(I.wwin + i), Yo[i] * e1[i]);
                });
                const int Mbc = Mcoarse / R;
                for (int n1 = tid; n1 < Mbc; n1 += T) {
                    const int pos = Swz<Rl>::f(n1);
                    const int m = p * Mbc + n1;
                    const cpx<Rl> e = d.tb[pos];
                    const double a = (double)e.x * inv * __ldg(I.twin + 2 * m);
                    const double b = (double)e.y * inv * __ldg(I.twin + 2 * m + 1);
                    d.tb[pos] = mk<Rl>((Rl)a, (Rl)b);
                }
                __syncthreads();
                dist_r2c<Rl, R>(d, Mcoarse, Nw, [&](int i, cpx<double> X) { Yo[i] = X; });
            }
            while (saved < I.saveN && I.zsave[saved] <= c.tn) {
                interpolate_row<Rl, Kt>(Nw, I.linop, c, I.zsave[saved], k, py, pyn,
                                        I.saves + (size_t)saved * Nw, p, R);
                ++saved;
            }
            swap_y = true;
        } else {
            cpx<double>* yn = reinterpret_cast<cpx<double>*>(pyn);
            for (int t = tid; own(t) < Nw; t += T) {
                const int i = own(t);
                yn[i] = y[i];
            }
            swap_y = false;
        }
    }
    __syncthreads();
    if (tid == 0 && writer) {
        I.status = c.status;
        I.steps = c.steps;
        I.nrhs = nrhs;
        I.nsaved = saved;
        I.z = c.tn;
        I.dz = c.dtn;
        I.y = py;
        I.yn = pyn;
        for (int j = 0; j < 7; ++j) I.k[j] = k[j];
    }
    // every CTA is done with the others' shared memory before the next instance starts
    dsync();
}

}  // namespace luna
