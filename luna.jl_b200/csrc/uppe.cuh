// Fused mode-averaged UPPE right-hand side and the interaction-picture RK45 loop,
// one instance per CTA.
//
// Right-hand side (NonlinearRHS.jl:362-373, TransModeAvg):
//   load E(omega) (fused with the RK stage combine and exp(L*dz))
//   -> zero-pad + inverse transform to the oversampled time grid (real: half-length
//      complex FFT with the split pre-twiddle; envelope: complex FFT)
//   -> responses accumulated in tuple order: Kerr, PlasmaCumtrapz (three block scans
//      for the cumulative integrals), Raman convolution on the 2x grid
//   -> time window -> forward transform -> crop, normalisation, frequency window
//   -> store (fused with exp(-L*dz) into the stage derivative).
//
// Integrator (RK45.jl:128-226, 249-297, 343-406 with dopri.jl) and Luna.run's per-step
// window filter and GridCondition saves (Luna.jl:366-372, Output.jl:65-82, 490-502).
#pragma once
#include "common.cuh"
#include "fft.cuh"
#include "inst.h"

namespace luna {

// ------------------------------------------------------------------ workspace layout
template <typename Rl>
struct Ws {
    cpx<Rl>* main;      // transform buffer
    cpx<Rl>* main_alt;  // second buffer (global memory only): out-of-place transforms
    cpx<Rl>* efac;      // exp(L*dz) of the current stage, Nw entries
    cpx<Rl>* ram;       // Raman convolution buffer (No complex)
    cpx<Rl>* ram_alt;
    cpx<Rl>* hil;       // Hilbert transform H of the field (no-THG responses), No/2 pairs
    cpx<Rl>* hil_alt;   // its out-of-place partner (global memory only)
    double* red;        // 3 * LUNA_WARPS reduction scratch
    double* tot;        // 3 * LUNA_WARPS scan totals
    double* edge;       // 4 edge values carried between scan chunks
    int* flag;          // status flags raised inside the RHS
    TwTab<Rl> tw;
    // Raman convolution on two helper CTAs of a thread-block cluster (rank 1: even,
    // rank 2: odd frequency half); null when the convolution runs in this CTA
    struct ClBox* cl;
    const cpx<Rl>* rem_e;  // helper buffers in distributed shared memory
    const cpx<Rl>* rem_o;
    const cpx<Rl>* rem_p;  // plasma polarisation from the plasma helper (rank 3)
};

// Mailbox of one CTA of a response cluster (static shared memory). Rank 0 writes the
// command fields of the helpers' boxes and then their `seq` (release); helper h writes
// `done[h-1]` of rank 0's box (release) when its part of the responses is ready.
#define CL_HELPERS 3
struct ClBox {
    int seq;
    int cmd;
    unsigned xaddr;  // shared-window offset of rank 0's field buffer
    int P;           // split factor of that buffer
    int M;           // pairs in that buffer (No/2)
    int inst;        // instance index
    float sc;        // field scale of the stored samples
    int done[CL_HELPERS];
    int pflag;       // status bits raised by the plasma helper's rate evaluations
};

#define CL_RAMAN 1
#define CL_EXIT 2

struct Ctl {  // controller state shared by the CTA (shared memory)
    void* k[7];  // stage derivative buffers (FSAL rotates k1 and k7)
    double t, tn, dt, dtn, err, errlast;
    int ok;
    int done;
    int status;
    int repeated;
    long long steps;
    int inst;
};

__host__ __device__ inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// main transform length (complex elements) for an instance
__host__ __device__ inline int main_len(const LunaInst& I) {
    int M = (I.kind == 0) ? I.No / 2 : I.No;
    int Mc = (I.kind == 0) ? I.N / 2 : I.N;
    return M > Mc ? M : Mc;
}

__host__ __device__ inline bool has_raman(const LunaInst& I) {
    for (int i = 0; i < I.nresp; ++i)
        if (I.resp[i].kind == LUNA_RESP_RAMAN) return true;
    return false;
}

// an instance with a no-THG response needs the Hilbert transform of its field
__host__ __device__ inline bool needs_hilbert(const LunaInst& I) {
    for (int i = 0; i < I.nresp; ++i)
        if (I.resp[i].hilb) return true;
    return false;
}

__host__ __device__ inline bool has_plasma(const LunaInst& I) {
    for (int i = 0; i < I.nresp; ++i)
        if (I.resp[i].kind == LUNA_RESP_PLASMA_PPT || I.resp[i].kind == LUNA_RESP_PLASMA_ADK) return true;
    return false;
}

// Bytes of global scratch an instance needs when nothing lives in shared memory.
template <typename Rl>
__host__ __device__ inline size_t gscr_bytes(const LunaInst& I) {
    size_t c = sizeof(cpx<Rl>);
    size_t b = 0;
    b += 2 * align_up((size_t)main_len(I) * c, 256);
    if (needs_hilbert(I)) b += 2 * align_up((size_t)(I.No / 2) * c, 256);
    b += align_up((size_t)I.Nw * c, 256);
    if (has_raman(I)) b += 2 * align_up((size_t)I.No * c, 256);
    return b;
}

#define LUNA_SMALL_BYTES 2048

template <typename Rl>
__device__ void plan_ws(const LunaInst& I, char* smem, int smem_bytes, Ws<Rl>& w, const TwTab<Rl>& tw,
                        void* gscr = nullptr, bool raman_remote = false) {
    w.cl = nullptr;
    w.rem_e = w.rem_o = w.rem_p = nullptr;
    w.red = reinterpret_cast<double*>(smem);
    w.tot = w.red + 3 * LUNA_WARPS;
    w.edge = w.tot + 3 * LUNA_WARPS;
    w.flag = reinterpret_cast<int*>(w.edge + 4);
    w.tw = tw;
    size_t off = LUNA_SMALL_BYTES;
    const size_t c = sizeof(cpx<Rl>);
    char* g = reinterpret_cast<char*>(gscr ? gscr : I.gscr);
    size_t goff = 0;
    const int Mm = main_len(I);
    size_t mb = align_up((size_t)Mm * c, 256);
    if (off + mb <= (size_t)smem_bytes) {
        w.main = reinterpret_cast<cpx<Rl>*>(smem + off);
        w.main_alt = nullptr;
        off += mb;
    } else {
        w.main = reinterpret_cast<cpx<Rl>*>(g + goff);
        w.main_alt = reinterpret_cast<cpx<Rl>*>(g + goff + mb);
    }
    goff += 2 * mb;
    w.hil = w.hil_alt = nullptr;
    if (needs_hilbert(I)) {
        const size_t hb = align_up((size_t)(I.No / 2) * c, 256);
        if (off + hb <= (size_t)smem_bytes) {
            w.hil = reinterpret_cast<cpx<Rl>*>(smem + off);
            off += hb;
        } else {
            w.hil = reinterpret_cast<cpx<Rl>*>(g + goff);
            w.hil_alt = reinterpret_cast<cpx<Rl>*>(g + goff + hb);
        }
        goff += 2 * hb;
    }
    size_t eb = align_up((size_t)I.Nw * c, 256);
    if (off + eb <= (size_t)smem_bytes) {
        w.efac = reinterpret_cast<cpx<Rl>*>(smem + off);
        off += eb;
    } else {
        w.efac = reinterpret_cast<cpx<Rl>*>(g + goff);
    }
    goff += eb;
    w.ram = w.ram_alt = nullptr;
    if (has_raman(I) && !raman_remote) {
        size_t rb = align_up((size_t)I.No * c, 256);
        if (off + rb <= (size_t)smem_bytes) {
            w.ram = reinterpret_cast<cpx<Rl>*>(smem + off);
            off += rb;
        } else {
            w.ram = reinterpret_cast<cpx<Rl>*>(g + goff);
            w.ram_alt = reinterpret_cast<cpx<Rl>*>(g + goff + rb);
        }
        goff += 2 * rb;
    }
}

// ------------------------------------------------------------------ block reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Deterministic block sum of three values; result valid in every thread.
__device__ __forceinline__ void block_sum3(double& a, double& b, double& c, double* red) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    __syncthreads();
    if (lane == 0) {
        red[wid] = a;
        red[LUNA_WARPS + wid] = b;
        red[2 * LUNA_WARPS + wid] = c;
    }
    __syncthreads();
    double sa = 0, sb = 0, sc = 0;
#pragma unroll
    for (int i = 0; i < LUNA_WARPS; ++i) {
        sa += red[i];
        sb += red[LUNA_WARPS + i];
        sc += red[2 * LUNA_WARPS + i];
    }
    a = sa;
    b = sb;
    c = sc;
}

// Block exclusive scan of one double per thread (one barrier). `tot` must not be
// reused by another scan before the next barrier that follows every thread's return.
__device__ __forceinline__ double block_exscan(double v, double* tot, double& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        double y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tot[wid] = x;
    __syncthreads();
    double off = 0, all = 0;
#pragma unroll
    for (int i = 0; i < LUNA_WARPS; ++i) {
        double tv = tot[i];
        off += (i < wid) ? tv : 0.0;
        all += tv;
    }
    total = all;
    return off + x - v;
}

// ------------------------------------------------------------------ rate functions
template <typename Rl>
__device__ __forceinline__ Rl ppt_rate(const LunaResp& r, Rl aE, int* flag);

template <>
__device__ __forceinline__ double ppt_rate<double>(const LunaResp& r, double aE, int* flag) {
    // Ionisation.jl:257-270 with CSpline evaluation (Maths.jl:835-848) and the uniform
    // index function (Maths.jl:772-774)
    if (aE < r.Emin) return 0.0;
    if (aE > r.Emax) {
        atomicOr(flag, 1 << ST_FIELD_ABOVE_EMAX);
        return 0.0;
    }
    const int n = r.sn;
    const double xmin = r.Emin, xmax = r.Emax;
    int i1;
    if (aE <= xmin) i1 = 2;
    else if (aE >= xmax) i1 = n;
    else i1 = (int)ceil((aE - xmin) / (xmax - xmin) * (double)(n - 1)) + 1;
    // already in [2, n] for every field inside the table; a NaN field (which passes both
    // range tests) would otherwise index before the table
    i1 = max(2, min(n, i1));
    const int i = i1 - 1;
    const double xi = __ldg(r.sx + i), xm = __ldg(r.sx + i - 1);
    const double yi = __ldg(r.sy + i), ym = __ldg(r.sy + i - 1);
    double v;
    if (aE == xi) v = yi;
    else if (aE == xm) v = ym;
    else {
        const double Di = __ldg(r.sD + i), Dm = __ldg(r.sD + i - 1);
        const double t = (aE - xm) / (xi - xm);
        v = ym + Dm * t + (3.0 * (yi - ym) - 2.0 * Dm - Di) * (t * t)
            + (2.0 * (ym - yi) + Dm + Di) * (t * t * t);
    }
    return exp(v);
}

template <>
__device__ __forceinline__ float ppt_rate<float>(const LunaResp& r, float aE, int* flag) {
    if (aE < (float)r.Emin) return 0.0f;
    if (aE > (float)r.Emax) {
        atomicOr(flag, 1 << ST_FIELD_ABOVE_EMAX);
        return 0.0f;
    }
    const int n = r.sn;
    const float xmin = (float)r.Emin, xmax = (float)r.Emax;
    int i1 = (int)ceilf((aE - xmin) / (xmax - xmin) * (float)(n - 1)) + 1;
    i1 = max(2, min(n, i1));
    const int i = i1 - 1;
    const float xi = __ldg(r.sxf + i), xm = __ldg(r.sxf + i - 1);
    const float yi = __ldg(r.syf + i), ym = __ldg(r.syf + i - 1);
    const float Di = __ldg(r.sDf + i), Dm = __ldg(r.sDf + i - 1);
    const float t = (aE - xm) / (xi - xm);
    const float v = ym + Dm * t + (3.0f * (yi - ym) - 2.0f * Dm - Di) * (t * t)
                    + (2.0f * (ym - yi) + Dm + Di) * (t * t * t);
    return expf(v);
}

template <typename Rl>
__device__ __forceinline__ Rl adk_rate(const LunaResp& r, Rl aE) {
    // Ionisation.jl:43-59: pre * (a/|E|)^(2n*-1) * exp(-b/|E|) above the threshold
    if (aE < (Rl)r.adk_thr || aE == (Rl)0) return (Rl)0;
    if (sizeof(Rl) == 8) {
        double x = (double)aE;
        return (Rl)(r.adk_pre * pow(r.adk_a / x, r.adk_pw) * exp(-r.adk_b / x));
    } else {
        float x = (float)aE;
        float lg = (float)r.adk_pw * logf((float)r.adk_a / x) - (float)r.adk_b / x + logf((float)r.adk_pre);
        return (Rl)expf(lg);
    }
}

template <typename Rl>
__device__ __forceinline__ Rl eval_rate(const LunaResp& r, Rl aE, int* flag) {
    return r.kind == LUNA_RESP_PLASMA_PPT ? ppt_rate<Rl>(r, aE, flag) : adk_rate<Rl>(r, aE);
}

// ------------------------------------------------------------------ real-FFT helpers
// exp(+-2*pi*i*k/(2M)) as a table twiddle
template <typename Rl, bool INV>
__device__ __forceinline__ cpx<double> half_twiddle(const TwTab<Rl>& tw, int k, int M) {
    const int shift = TW_LOG_MMAX - (ilog2i((unsigned)M) + 1);
    cpx<Rl> w = twiddle<Rl, INV>(tw, (unsigned)k << shift);
    return cvt<double>(w);
}

// Raman convolution on the 2*No grid (Nonlinear.jl:282-333): the input samples s[n]
// (n < No) are in `ram` as complex pairs (s[2m], s[2m+1]) for m < No/2 (zero above), in
// split order; on return `ram` holds P[n], n < No, as pairs in split order.
// Returns the buffer that holds P (w.ram or, out of place, w.ram_alt).
template <typename Rl>
__device__ __forceinline__ cpx<Rl>* raman_conv(const LunaResp& r, int No, Ws<Rl>& w) {
    __syncthreads();
    cpx<Rl>* Z = block_fft<Rl, false>(w.ram, w.ram_alt, No, w.tw);
    const cpx<Rl>* H = reinterpret_cast<const cpx<Rl>*>(r.H);
    const int M = No;  // complex length of the 2*No real transform
    for (int k = threadIdx.x; k <= M / 2; k += LUNA_BLOCK) {
        const int km = (M - k) & (M - 1);
        cpx<double> Zk = cvt<double>(Z[Swz<Rl>::f(k)]);
        cpx<double> Zm = cvt<double>(Z[Swz<Rl>::f(km)]);
        // forward split: X[k] = 1/2 (Z[k] + conj Z[M-k]) - i/2 W^k (Z[k] - conj Z[M-k])
        cpx<double> Wk = half_twiddle<Rl, false>(w.tw, k, M);
        cpx<double> a = Zk + conj(Zm), b = Zk - conj(Zm);
        cpx<double> Xk = scale(0.5, a) + scale(0.5, mul_mi<double, false>(Wk * b));
        cpx<double> Xm;  // X[M-k]
        if (k == 0) {
            Xk = mk<double>(Zk.x + Zk.y, 0.0);
            Xm = mk<double>(Zk.x - Zk.y, 0.0);  // X[M]
        } else {
            // W^(M-k) = -conj(W^k)
            cpx<double> Wm = scale(-1.0, conj(Wk));
            cpx<double> a2 = Zm + conj(Zk), b2 = Zm - conj(Zk);
            Xm = scale(0.5, a2) + scale(0.5, mul_mi<double, false>(Wm * b2));
        }
        // a spectrum rebuilt at rho(z) by this kernel is read with plain loads
        const cpx<double> Hk = r.hz ? cvt<double>(H[k]) : cvt<double>(ldg(H + k));
        const cpx<double> Hm = r.hz ? cvt<double>(H[M - k]) : cvt<double>(ldg(H + (M - k)));
        cpx<double> Yk = Xk * Hk;
        cpx<double> Ym = Xm * Hm;
        // inverse split: Z'[k] = (Y[k] + conj Y[M-k]) + i W^-k (Y[k] - conj Y[M-k])
        cpx<double> Wi = conj(Wk);
        cpx<double> Zk2 = (Yk + conj(Ym)) + mul_mi<double, true>(Wi * (Yk - conj(Ym)));
        Z[Swz<Rl>::f(k)] = cvt<Rl>(Zk2);
        if (k != 0 && km != k) {
            cpx<double> Wmi = scale(-1.0, Wk);  // W^-(M-k) = -W^k
            cpx<double> Zm2 = (Ym + conj(Yk)) + mul_mi<double, true>(Wmi * (Ym - conj(Yk)));
            Z[Swz<Rl>::f(km)] = cvt<Rl>(Zm2);
        }
    }
    __syncthreads();
    cpx<Rl>* other = w.ram_alt ? ((Z == w.ram) ? w.ram_alt : w.ram) : nullptr;
    return block_fft<Rl, true>(Z, other, No, w.tw);
}

// Dephasing time of Raman component c at density rho (Raman.jl:142-157, 229-238): the laws
// of luna_resp_desc.tau2_rho in the reference's order of operations, each rounded.
__device__ __forceinline__ double raman_tau2(const LunaResp& r, int c, double rho) {
    const double* q = r.t2rho + 4 * c;
    const int model = (int)q[0];
    if (model == 0) return r.tau2[c];
    if (model == 1 && !(rho > 0)) return INFINITY;
    const double s = __dadd_rn(__dadd_rn(model == 2 ? q[3] : 0.0, __ddiv_rn(q[1], __ddiv_rn(rho, r.amg))),
                               __ddiv_rn(__dmul_rn(q[2], rho), r.amg));
    return __ddiv_rn(1.0, __dmul_rn(3.141592653589793, s));  // π as a double
}

// hscale * h(t_n; tau2) of a Raman response (CombinedRamanResponse(ht, rho), Raman.jl:256-262):
// w(t_n) * sum_c hpre_c(t_n) exp(-t_n / tau2_c). The damping at t = 0 is 1 for every tau2,
// including tau2 = 0 (a vibrational law at rho = 0, where the reference forms 0/0; its
// undamped response is 0 there, and the polarisation is scaled by rho = 0).
__device__ __forceinline__ double raman_sample(const LunaResp& r, int No, int n, const double* tau2, double hscale) {
    const double tt = r.htt[n];
    double h = 0;
    for (int c = 0; c < r.ncomp; ++c) h += r.hpre[(size_t)c * No + n] * (tt == 0.0 ? 1.0 : exp(-tt / tau2[c]));
    return h * (r.hwin[n] * hscale);
}

// Raman response spectrum at density rho for a plan with a pressure gradient whose
// dephasing times depend on the density; the reference rebuilds h(t; rho) and transforms it
// at every call (Nonlinear.jl:306-307). Samples as raman_h_kernel, transformed in the compute
// precision in the Raman buffers (free between evaluations) into the writable r.H.
template <typename Rl>
__device__ __noinline__ void raman_h_at(const LunaInst& I, Ws<Rl>& w, double rho) {
    const LunaResp& r = I.resp[I.ramz - 1];
    const int No = I.No, tid = threadIdx.x;
    double t2[LUNA_RAMAN_MAXC];
#pragma unroll
    for (int c = 0; c < LUNA_RAMAN_MAXC; ++c) t2[c] = (c < r.ncomp) ? raman_tau2(r, c, rho) : 1.0;
    const int P = buf_split<Rl>(w.ram_alt, No);
    __syncthreads();
    for (int m = tid; m < No; m += LUNA_BLOCK) {
        double a = 0, b = 0;
        if (m < No / 2) {
            a = raman_sample(r, No, 2 * m, t2, r.hscale);
            b = raman_sample(r, No, 2 * m + 1, t2, r.hscale);
        }
        w.ram[Swz<Rl>::f(split_pos(m, No, P))] = mk<Rl>((Rl)a, (Rl)b);
    }
    __syncthreads();
    const cpx<Rl>* Z = block_fft<Rl, false>(w.ram, w.ram_alt, No, w.tw);
    cpx<Rl>* H = reinterpret_cast<cpx<Rl>*>(const_cast<void*>(r.H));
    const int M = No;
    for (int k = tid; k <= M; k += LUNA_BLOCK) {
        const cpx<double> Zk = cvt<double>(Z[Swz<Rl>::f(k & (M - 1))]);
        const cpx<double> Zm = cvt<double>(Z[Swz<Rl>::f((M - k) & (M - 1))]);
        cpx<double> X;
        if (k == 0) X = mk<double>(Zk.x + Zk.y, 0.0);
        else if (k == M) X = mk<double>(Zk.x - Zk.y, 0.0);
        else {
            const cpx<double> Wk = half_twiddle<Rl, false>(w.tw, k, M);
            X = scale(0.5, Zk + conj(Zm)) + scale(0.5, mul_mi<double, false>(Wk * (Zk - conj(Zm))));
        }
        H[k] = cvt<Rl>(X);
    }
    __syncthreads();
}

// ------------------------------------------------------------------ Raman clusters
#define CL_WAIT_CYCLES (4000000000LL)  // ~2 s at the B200 boost clock

__device__ __forceinline__ unsigned cl_map(const void* p, unsigned rank) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
    return r;
}
__device__ __forceinline__ void cl_st(unsigned caddr, unsigned v) {
    asm volatile("st.shared::cluster.u32 [%0], %1;" ::"r"(caddr), "r"(v) : "memory");
}
__device__ __forceinline__ void cl_st_release(unsigned caddr, unsigned v) {
    asm volatile("st.release.cluster.shared::cluster.u32 [%0], %1;" ::"r"(caddr), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned cl_ld_acquire(const void* p) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(p);
    unsigned v;
    asm volatile("ld.acquire.cluster.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(a) : "memory");
    return v;
}
__device__ __forceinline__ void cl_fence() { asm volatile("fence.acq_rel.cluster;" ::: "memory"); }

// Rank 0 of a response cluster: post the field buffer x (shared memory, split factor P)
// to the helpers and wait, bounded, until the two Raman halves and the plasma
// polarisation are in their shared memory. False after a timeout (or once the cluster is
// marked broken): the caller then drops those terms and raises ST_WAIT_TIMEOUT, and no
// further command is posted.
template <typename Rl>
__device__ bool cluster_post_wait(Ws<Rl>& w, const cpx<Rl>* x, int M, int P, double sc, int inst) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ClBox* box = w.cl;
        int ok = box->cmd != -1;  // -1 marks a broken cluster
        if (ok) {
            const int seq = ++box->seq;
            const unsigned xa = (unsigned)__cvta_generic_to_shared(x);
            for (unsigned h = 1; h <= CL_HELPERS; ++h) {
                cl_st(cl_map(&box->cmd, h), CL_RAMAN);
                cl_st(cl_map(&box->xaddr, h), xa);
                cl_st(cl_map(&box->P, h), (unsigned)P);
                cl_st(cl_map(&box->M, h), (unsigned)M);
                cl_st(cl_map(&box->inst, h), (unsigned)inst);
                cl_st(cl_map(&box->sc, h), __float_as_uint((float)sc));
            }
            cl_fence();
            for (unsigned h = 1; h <= CL_HELPERS; ++h) cl_st_release(cl_map(&box->seq, h), (unsigned)seq);
            const long long t0 = clock64();
            while (true) {
                bool all = true;
                for (int h = 0; h < CL_HELPERS; ++h) all = all && ((int)cl_ld_acquire(&box->done[h]) == seq);
                if (all) break;
                if (clock64() - t0 > CL_WAIT_CYCLES) {
                    ok = 0;
                    box->cmd = -1;
                    break;
                }
            }
            if (ok && box->pflag) atomicOr(w.flag, box->pflag);
        }
        if (!ok) atomicOr(w.flag, 1 << ST_WAIT_TIMEOUT);
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// ------------------------------------------------------------------ plasma chunk
// Running integrals carried from one chunk of samples to the next.
struct PlasmaCarry {
    double c1, c2, c3;
};

// PlasmaScalar! (Nonlinear.jl:121-133) for the two consecutive pairs (samples 4t..4t+3 of
// a chunk of 4*LUNA_BLOCK samples) held by this thread. Each running trapezoid is written
// as dt*(prefix_sum(y)[n] - (y[0]+y[n])/2), so the three cumulative integrals are block
// prefix sums (FP64) of the thread's four samples summed in order, carried across chunks;
// y[0] of each integrand is broadcast from the first chunk through `edge`.
template <typename Rl>
__device__ __forceinline__ void plasma_quad(const LunaResp& r, const bool act[2], int m0, const double E[4],
                                            PlasmaCarry& cr, Ws<Rl>& w, double Pq[4]) {
    const double dt = r.dt, er = r.eratio;
    double rr[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) rr[s] = act[s >> 1] ? (double)eval_rate<Rl>(r, (Rl)fabs(E[s]), w.flag) : 0.0;
    if (m0 == 0) w.edge[0] = rr[0];
    double tot;
    double x = block_exscan(((rr[0] + rr[1]) + rr[2]) + rr[3], w.tot, tot);
    const double y0r = w.edge[0];
    double S = cr.c1 + x;
    cr.c1 += tot;
    double fr[4], ph[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        S += rr[s];
        const double f = dt * (S - 0.5 * (y0r + rr[s]));
        fr[s] = r.preion + 1.0 - ((f == 0.0) ? 1.0 : exp(-f));
        ph[s] = act[s >> 1] ? fr[s] * er * E[s] : 0.0;
    }
    if (m0 == 0) w.edge[1] = ph[0];
    x = block_exscan(((ph[0] + ph[1]) + ph[2]) + ph[3], w.tot + LUNA_WARPS, tot);
    const double y0p = w.edge[1];
    double T = cr.c2 + x;
    cr.c2 += tot;
    double J[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        T += ph[s];
        J[s] = dt * (T - 0.5 * (y0p + ph[s]));
        if (act[s >> 1] && fabs(E[s]) > 0) J[s] += r.ionpot * rr[s] * (1.0 - fr[s]) / E[s];
        if (!act[s >> 1]) J[s] = 0;
    }
    if (m0 == 0) w.edge[2] = J[0];
    x = block_exscan(((J[0] + J[1]) + J[2]) + J[3], w.tot + 2 * LUNA_WARPS, tot);
    const double y0J = w.edge[2];
    double U = cr.c3 + x;
    cr.c3 += tot;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        U += J[s];
        Pq[s] += r.coef * (dt * (U - 0.5 * (y0J + J[s])));
    }
}

// Plasma polarisation alone, for the plasma helper of a response cluster: the field is
// read from xr (rank 0's buffer, split factor P) and rho * P_plasma is written to out at
// the same positions.
template <typename Rl>
__device__ void plasma_only(const LunaInst& I, Ws<Rl>& w, const cpx<Rl>* xr, cpx<Rl>* out, int M, int P, double sc,
                            int ip) {
    const int T = LUNA_BLOCK, tid = threadIdx.x;
    PlasmaCarry cr = {0, 0, 0};
    // the remote field of the next chunk is loaded while the current one is processed
    cpx<Rl> nx[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int m = 2 * tid + q;
        nx[q] = (m < M) ? xr[Swz<Rl>::f(split_pos(m, M, P))] : mk<Rl>(0, 0);
    }
    for (int c0 = 0; c0 < M; c0 += 2 * T) {
        const int m0 = c0 + 2 * tid;
        const bool act[2] = {m0 < M, m0 + 1 < M};
        int pos[2];
        double E[4];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            pos[q] = Swz<Rl>::f(split_pos(act[q] ? m0 + q : 0, M, P));
            const cpx<Rl> e = act[q] ? nx[q] : mk<Rl>(0, 0);
            E[2 * q] = (double)e.x * sc;
            E[2 * q + 1] = (double)e.y * sc;
            const int mn = m0 + 2 * T + q;
            nx[q] = (mn < M) ? xr[Swz<Rl>::f(split_pos(mn, M, P))] : mk<Rl>(0, 0);
        }
        double Pq[4] = {0, 0, 0, 0};
        plasma_quad<Rl>(I.resp[ip], act, m0, E, cr, w, Pq);
#pragma unroll
        for (int q = 0; q < 2; ++q)
            if (act[q]) out[pos[q]] = mk<Rl>((Rl)Pq[2 * q], (Rl)Pq[2 * q + 1]);
    }
    __syncthreads();
}

// ------------------------------------------------------------------ the right-hand sides
// load(k) -> cpx<double> input bin k (k < Nw); store(k, v) consumes output bin k (k < Nw).

// field-resolved grid (RealGrid): to_time! / to_freq! with rfft semantics, in three
// phases that the radial transform reuses per column.

// to_time! (NonlinearRHS.jl:16-23): C2R pre-twiddle of the zero-padded spectrum and the
// inverse transform. Returns the buffer holding slot m = samples (2m, 2m+1) in split
// order with factor *P (unscaled: multiply by the pad scale / No).
//
// With hx != null the same pass also transforms the spectrum -i X[k] (k >= 1; DC and
// Nyquist zero) into w.hil: the Hilbert transform H of the field, so that the analytic
// signal of Maths.hilbert (Maths.jl:560-569) is E + iH (the padded spectrum is zero at
// the Nyquist bin, so its real part is E itself). *hx receives the buffer holding H in
// split order with factor *Ph, scaled like E.
template <typename Rl, typename LoadF>
__device__ __forceinline__ cpx<Rl>* c2r_to_time(Ws<Rl>& w, int M, int Nw, LoadF&& load, int* P,
                                                cpx<Rl>** hx = nullptr, int* Ph = nullptr) {
    const int T = LUNA_BLOCK;
    const int tid = threadIdx.x;
    cpx<Rl>* buf = w.main;
    cpx<Rl>* hb = hx ? w.hil : nullptr;
    // Z[k] = (X[k] + conj X[M-k]) + i W^-k (X[k] - conj X[M-k])
    for (int k = tid; k <= M / 2; k += T) {
        const int km = M - k;
        cpx<double> Xk = (k < Nw) ? load(k) : mk<double>(0, 0);
        // each bin is loaded once (the loader may update stage state in place)
        cpx<double> Xm = (km == k) ? Xk : ((km < Nw) ? load(km) : mk<double>(0, 0));
        if (k == 0) {  // imaginary parts of DC and Nyquist do not enter a real transform
            Xk.y = 0;
            Xm.y = 0;
        }
        cpx<double> Wi = half_twiddle<Rl, true>(w.tw, k, M);
        cpx<double> Zk = (Xk + conj(Xm)) + mul_mi<double, true>(Wi * (Xk - conj(Xm)));
        buf[Swz<Rl>::f(k)] = cvt<Rl>(Zk);
        if (k != 0 && km != k) {
            cpx<double> Wmi = scale(-1.0, conj(Wi));
            cpx<double> Zm = (Xm + conj(Xk)) + mul_mi<double, true>(Wmi * (Xm - conj(Xk)));
            buf[Swz<Rl>::f(km)] = cvt<Rl>(Zm);
        }
        if (hb) {
            // -i X (DC and Nyquist bins dropped, as the analytic signal does)
            const cpx<double> Hk = (k == 0) ? mk<double>(0, 0) : mk<double>(Xk.y, -Xk.x);
            const cpx<double> Hm = (k == 0) ? mk<double>(0, 0) : mk<double>(Xm.y, -Xm.x);
            hb[Swz<Rl>::f(k)] = cvt<Rl>((Hk + conj(Hm)) + mul_mi<double, true>(Wi * (Hk - conj(Hm))));
            if (k != 0 && km != k) {
                cpx<double> Wmi = scale(-1.0, conj(Wi));
                hb[Swz<Rl>::f(km)] = cvt<Rl>((Hm + conj(Hk)) + mul_mi<double, true>(Wmi * (Hm - conj(Hk))));
            }
        }
    }
    __syncthreads();
    cpx<Rl>* x = block_fft<Rl, true>(buf, w.main_alt, M, w.tw);
    *P = buf_split<Rl>(w.main_alt, M);
    if (hb) {
        *hx = block_fft<Rl, true>(hb, w.hil_alt, M, w.tw);
        *Ph = buf_split<Rl>(w.hil_alt, M);
    }
    return x;
}

// Et_to_Pt! (NonlinearRHS.jl:121-126) and the time window, in place on the samples held
// by x (split factor P); sc converts the stored samples to the field in V/m. hx (split
// factor Ph) holds the Hilbert transform of the field for the no-THG responses, whose
// squared field is |hilbert(E)|^2 = E^2 + H^2 (Kerr_field_nothg: 3/4 coef (E^2 + H^2) E,
// Nonlinear.jl:36-45; RamanPolarField(thg=false): 1/2 (E^2 + H^2), Nonlinear.jl:267-275).
// HIL selects the no-THG variant at compile time, so that the THG forms (the common case)
// compile to the same code as without it.
template <typename Rl, bool HIL>
__device__ __forceinline__ void pointwise_real_t(const LunaInst& I, Ws<Rl>& w, cpx<Rl>* x, int M, int P, double sc,
                                                 const cpx<Rl>* hx, int Ph) {
    const int T = LUNA_BLOCK;
    const int tid = threadIdx.x;
    int ip = -1, ir = -1;
    for (int i = 0; i < I.nresp; ++i) {
        if (I.resp[i].kind == LUNA_RESP_PLASMA_PPT || I.resp[i].kind == LUNA_RESP_PLASMA_ADK) ip = i;
        if (I.resp[i].kind == LUNA_RESP_RAMAN) ir = i;
    }
    const int Pr_split = (ir >= 0) ? buf_split<Rl>(w.ram_alt, I.No) : 1;
    cpx<Rl>* Pr = nullptr;
    if (!HIL && w.cl) {
        // response cluster: Raman halves on ranks 1-2 (P_raman[m] = even[m] + odd[m] in
        // the split order of their No/2-point transforms), plasma polarisation on rank 3
        // (same positions as x); the responses are added here in tuple order
        const bool ok = cluster_post_wait<Rl>(w, x, M, P, sc, w.cl->inst);
        const int Ph = fft_nsplit<Rl>(M);
        const bool use_r = ok && ir >= 0, use_p = ok && ip >= 0;
        // four samples pairs per thread and round: every load of a round (own buffer,
        // helpers' shared memory, time window) is issued before the arithmetic
        constexpr int U = 4;
        for (int m0 = tid; m0 < M; m0 += U * T) {
            int pos[U];
            cpx<Rl> e[U], pr[U], pl[U];
            double2 tw[U];
#pragma unroll
            for (int q = 0; q < U; ++q) {
                const int m = m0 + q * T;
                const bool a = m < M;
                pos[q] = Swz<Rl>::f(split_pos(a ? m : 0, M, P));
                const int ph = Swz<Rl>::f(split_pos(a ? m : 0, M, Ph));
                e[q] = x[pos[q]];
                pr[q] = use_r ? w.rem_e[ph] + w.rem_o[ph] : mk<Rl>(0, 0);
                pl[q] = use_p ? w.rem_p[pos[q]] : mk<Rl>(0, 0);
                tw[q] = __ldg(reinterpret_cast<const double2*>(I.towin) + (a ? m : 0));
            }
#pragma unroll
            for (int q = 0; q < U; ++q) {
                if (m0 + q * T >= M) continue;
                const double E0 = (double)e[q].x * sc, E1 = (double)e[q].y * sc;
                double P0 = 0, P1 = 0;
                for (int i = 0; i < I.nresp; ++i) {
                    const LunaResp& r = I.resp[i];
                    if (r.kind == LUNA_RESP_KERR_FIELD) {
                        P0 += r.coef * (E0 * E0 * E0);
                        P1 += r.coef * (E1 * E1 * E1);
                    } else if (i == ir && use_r) {
                        P0 += r.coef * E0 * (double)pr[q].x;
                        P1 += r.coef * E1 * (double)pr[q].y;
                    } else if (i == ip && use_p) {
                        P0 += (double)pl[q].x;
                        P1 += (double)pl[q].y;
                    }
                }
                x[pos[q]] = mk<Rl>((Rl)(P0 * tw[q].x), (Rl)(P1 * tw[q].y));
            }
        }
        __syncthreads();
        return;
    }
    if (ir >= 0) {
        // E^2 (thg=true form of sqr!) or 1/2 (E^2 + H^2) (thg=false) on the first half of
        // the 2*No grid, split order
        const bool hq = HIL && I.resp[ir].hilb;
        for (int m = tid; m < I.No; m += T) {
            cpx<Rl> v = mk<Rl>(0, 0);
            if (m < M) {
                cpx<Rl> e = x[Swz<Rl>::f(split_pos(m, M, P))];
                Rl e0 = e.x * (Rl)sc, e1 = e.y * (Rl)sc;
                v = mk<Rl>(e0 * e0, e1 * e1);
                if constexpr (HIL) {
                    if (hq) {
                        const cpx<Rl> h = hx[Swz<Rl>::f(split_pos(m, M, Ph))];
                        const Rl h0 = h.x * (Rl)sc, h1 = h.y * (Rl)sc;
                        v = mk<Rl>((Rl)0.5 * (e0 * e0 + h0 * h0), (Rl)0.5 * (e1 * e1 + h1 * h1));
                    }
                }
            }
            w.ram[Swz<Rl>::f(split_pos(m, I.No, Pr_split))] = v;
        }
        Pr = raman_conv<Rl>(I.resp[ir], I.No, w);
    }
    PlasmaCarry cr = {0, 0, 0};
    if (ip >= 0) {
        // chunks of 2*T pairs, two consecutive pairs per thread
        for (int c0 = 0; c0 < M; c0 += 2 * T) {
            const int m0 = c0 + 2 * tid;
            const bool act[2] = {m0 < M, m0 + 1 < M};
            int pos[2];
            double E[4], H2[4] = {0, 0, 0, 0};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                pos[q] = Swz<Rl>::f(split_pos(act[q] ? m0 + q : 0, M, P));
                const cpx<Rl> e = act[q] ? x[pos[q]] : mk<Rl>(0, 0);
                E[2 * q] = (double)e.x * sc;
                E[2 * q + 1] = (double)e.y * sc;
                if constexpr (HIL) {
                    const cpx<Rl> h = act[q] ? hx[Swz<Rl>::f(split_pos(m0 + q, M, Ph))] : mk<Rl>(0, 0);
                    H2[2 * q] = (double)h.x * sc * ((double)h.x * sc);
                    H2[2 * q + 1] = (double)h.y * sc * ((double)h.y * sc);
                }
            }
            double Pq[4] = {0, 0, 0, 0};
            for (int i = 0; i < I.nresp; ++i) {
                const LunaResp& r = I.resp[i];
                if (HIL && r.kind == LUNA_RESP_KERR_FIELD && r.hilb) {
#pragma unroll
                    for (int s = 0; s < 4; ++s) Pq[s] += 0.75 * r.coef * (E[s] * E[s] + H2[s]) * E[s];
                } else if (r.kind == LUNA_RESP_KERR_FIELD) {
#pragma unroll
                    for (int s = 0; s < 4; ++s) Pq[s] += r.coef * (E[s] * E[s] * E[s]);
                } else if (i == ir) {
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const int m = m0 + q;
                        const cpx<Rl> pr = act[q] ? Pr[Swz<Rl>::f(split_pos(m, I.No, Pr_split))] : mk<Rl>(0, 0);
                        Pq[2 * q] += r.coef * E[2 * q] * (double)pr.x;
                        Pq[2 * q + 1] += r.coef * E[2 * q + 1] * (double)pr.y;
                    }
                } else if (i == ip) {
                    plasma_quad<Rl>(r, act, m0, E, cr, w, Pq);
                }
            }
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!act[q]) continue;
                const int m = m0 + q;
                const double tw0 = __ldg(I.towin + 2 * m), tw1 = __ldg(I.towin + 2 * m + 1);
                x[pos[q]] = mk<Rl>((Rl)(Pq[2 * q] * tw0), (Rl)(Pq[2 * q + 1] * tw1));
            }
        }
        __syncthreads();
        return;
    }
    for (int c0 = 0; c0 < M; c0 += T) {
        const int m = c0 + tid;
        const bool act = m < M;
        const int pos = Swz<Rl>::f(split_pos(m, M, P));
        cpx<Rl> e = act ? x[pos] : mk<Rl>(0, 0);
        const double E0 = (double)e.x * sc, E1 = (double)e.y * sc;
        double Hq0 = 0, Hq1 = 0;
        if constexpr (HIL) {
            const cpx<Rl> h = act ? hx[Swz<Rl>::f(split_pos(m, M, Ph))] : mk<Rl>(0, 0);
            Hq0 = (double)h.x * sc * ((double)h.x * sc);
            Hq1 = (double)h.y * sc * ((double)h.y * sc);
        }
        double P0 = 0, P1 = 0;
        for (int i = 0; i < I.nresp; ++i) {
            const LunaResp& r = I.resp[i];
            if (HIL && r.kind == LUNA_RESP_KERR_FIELD && r.hilb) {
                P0 += 0.75 * r.coef * (E0 * E0 + Hq0) * E0;
                P1 += 0.75 * r.coef * (E1 * E1 + Hq1) * E1;
            } else if (r.kind == LUNA_RESP_KERR_FIELD) {
                P0 += r.coef * (E0 * E0 * E0);
                P1 += r.coef * (E1 * E1 * E1);
            } else if (i == ir) {
                cpx<Rl> p = act ? Pr[Swz<Rl>::f(split_pos(m, I.No, Pr_split))] : mk<Rl>(0, 0);
                P0 += r.coef * E0 * (double)p.x;
                P1 += r.coef * E1 * (double)p.y;
            }
        }
        if (act) {
            const double tw0 = __ldg(I.towin + 2 * m), tw1 = __ldg(I.towin + 2 * m + 1);
            x[pos] = mk<Rl>((Rl)(P0 * tw0), (Rl)(P1 * tw1));
        }
    }
    __syncthreads();
}

template <typename Rl>
__device__ __forceinline__ void pointwise_real(const LunaInst& I, Ws<Rl>& w, cpx<Rl>* x, int M, int P, double sc) {
    pointwise_real_t<Rl, false>(I, w, x, M, P, sc, nullptr, 1);
}

// the no-THG variant, out of line: it adds the Hilbert samples to every path
template <typename Rl>
__device__ __noinline__ void pointwise_real_hilb(const LunaInst& I, Ws<Rl>& w, cpx<Rl>* x, int M, int P, double sc,
                                                 const cpx<Rl>* hx, int Ph) {
    pointwise_real_t<Rl, true>(I, w, x, M, P, sc, hx, Ph);
}

// to_freq! (NonlinearRHS.jl:39-45): forward transform of x (split factor of the buffer),
// R2C split X[k] = 1/2 (Z[k] + conj Z[M-k]) - i/2 W^k (Z[k] - conj Z[M-k]), crop to Nw,
// and hand bin k to store.
template <typename Rl, typename StoreF>
__device__ __forceinline__ void r2c_to_freq(Ws<Rl>& w, cpx<Rl>* x, int M, int Nw, StoreF&& store) {
    const int T = LUNA_BLOCK;
    const int tid = threadIdx.x;
    cpx<Rl>* Z = block_fft<Rl, false>(x, w.main_alt ? ((x == w.main) ? w.main_alt : w.main) : nullptr, M, w.tw);
    for (int k = tid; k < Nw; k += T) {
        const int km = (M - k) & (M - 1);
        cpx<double> Zk = cvt<double>(Z[Swz<Rl>::f(k & (M - 1))]);
        cpx<double> Zm = cvt<double>(Z[Swz<Rl>::f(km)]);
        cpx<double> X;
        if (k == 0) X = mk<double>(Zk.x + Zk.y, 0.0);
        else if (k == M) X = mk<double>(Zk.x - Zk.y, 0.0);
        else {
            cpx<double> Wk = half_twiddle<Rl, false>(w.tw, k, M);
            X = scale(0.5, Zk + conj(Zm)) + scale(0.5, mul_mi<double, false>(Wk * (Zk - conj(Zm))));
        }
        store(k, X);
    }
    __syncthreads();
}

template <typename Rl, typename LoadF, typename StoreF>
__device__ __forceinline__ void rhs_real(const LunaInst& I, Ws<Rl>& w, LoadF&& load, StoreF&& store) {
    const int M = I.No / 2;
    int P, Ph = 1;
    cpx<Rl>* hx = nullptr;
    cpx<Rl>* x = c2r_to_time<Rl>(w, M, I.Nw, load, &P, w.hil ? &hx : nullptr, &Ph);
    // field scale 1/(nlscale sqrt(Aeff)) x pad/No; a taper's is in outz[Nw] at this node
    const double sc = I.grad ? I.outz[I.Nw].x : I.in_scale;
    if (hx) pointwise_real_hilb<Rl>(I, w, x, M, P, sc, hx, Ph);
    else pointwise_real<Rl>(I, w, x, M, P, sc);
    const cpx<double>* of = reinterpret_cast<const cpx<double>*>(I.outfac);
    // with a pressure gradient the factor of the current z is in outz, written by this
    // kernel (plain loads, not the read-only path)
    const cpx<double>* oz = reinterpret_cast<const cpx<double>*>(I.outz);
    const bool zdep = I.grad != nullptr;
    r2c_to_freq<Rl>(w, x, M, I.Nw, [&](int k, cpx<double> X) { store(k, X * (zdep ? oz[k] : ldg(of + k))); });
}

// Et_to_Pt! and the time window for an envelope on the CTA's time buffer x (No complex
// samples in split order P, field = sc * x): Kerr_env, Kerr_env_thg and RamanPolarEnv
// (Nonlinear.jl:47-84, 296-333), in place.
template <typename Rl>
__device__ __noinline__ void pointwise_env(const LunaInst& I, Ws<Rl>& w, cpx<Rl>* x, int P, double sc) {
    const int No = I.No;
    const int T = LUNA_BLOCK;
    const int tid = threadIdx.x;
    int ir = -1;
    for (int i = 0; i < I.nresp; ++i)
        if (I.resp[i].kind == LUNA_RESP_RAMAN) ir = i;
    const int Pr_split = (ir >= 0) ? buf_split<Rl>(w.ram_alt, No) : 1;
    cpx<Rl>* Pr = nullptr;
    if (ir >= 0) {
        // 1/2 |E|^2 on the first half of the 2*No grid (sqr! for RamanPolarEnv), split order
        for (int m = tid; m < No; m += T) {
            cpx<Rl> v = mk<Rl>(0, 0);
            if (m < No / 2) {
                cpx<double> a = scale(sc, cvt<double>(x[Swz<Rl>::f(split_pos(2 * m, No, P))]));
                cpx<double> b = scale(sc, cvt<double>(x[Swz<Rl>::f(split_pos(2 * m + 1, No, P))]));
                v = mk<Rl>((Rl)(0.5 * abs2(a)), (Rl)(0.5 * abs2(b)));
            }
            w.ram[Swz<Rl>::f(split_pos(m, No, Pr_split))] = v;
        }
        Pr = raman_conv<Rl>(I.resp[ir], No, w);
    }
    for (int n = tid; n < No; n += T) {
        const int pos = Swz<Rl>::f(split_pos(n, No, P));
        cpx<double> E = scale(sc, cvt<double>(x[pos]));
        cpx<double> Pt = mk<double>(0, 0);
        for (int i = 0; i < I.nresp; ++i) {
            const LunaResp& r = I.resp[i];
            if (r.kind == LUNA_RESP_KERR_ENV && r.cthg) {
                // Kerr_env_thg (Nonlinear.jl:75-84): coef/4 (3|E|^2 + exp(2i w0 t) E^2) E
                const cpx<double> C = ldg(reinterpret_cast<const cpx<double>*>(r.cthg) + n);
                Pt = Pt + scale(0.25 * r.coef, scale(3.0 * abs2(E), E) + C * (E * E) * E);
            } else if (r.kind == LUNA_RESP_KERR_ENV) {
                Pt = Pt + scale(0.75 * r.coef * abs2(E), E);
            } else if (i == ir) {
                cpx<Rl> p = Pr[Swz<Rl>::f(split_pos(n >> 1, No, Pr_split))];
                double pv = (n & 1) ? (double)p.y : (double)p.x;
                Pt = Pt + scale(r.coef * pv, E);
            }
        }
        x[pos] = cvt<Rl>(scale(__ldg(I.towin + n), Pt));
    }
    __syncthreads();
}

// envelope grid: to_time! of an Nw-bin spectrum with copy_scale_both! padding (the pad
// scale is in the field scale), as No complex time samples in split order; returns the
// buffer that holds them and their split factor in *P
template <typename Rl, typename LoadF>
__device__ __forceinline__ cpx<Rl>* env_to_time(const LunaInst& I, Ws<Rl>& w, LoadF&& load, int* P) {
    const int No = I.No, N = I.N, h = I.N / 2;
    cpx<Rl>* buf = w.main;
    for (int j = threadIdx.x; j < No; j += LUNA_BLOCK) {
        cpx<double> X = mk<double>(0, 0);
        if (j < h) X = load(j);
        else if (j >= No - h) X = load(j - No + N);
        buf[Swz<Rl>::f(j)] = cvt<Rl>(X);
    }
    __syncthreads();
    *P = buf_split<Rl>(w.main_alt, No);
    return block_fft<Rl, true>(buf, w.main_alt, No, w.tw);  // E(t), split order
}

// envelope grid: to_freq! of the time buffer x (split order) into store(k, X), k < N
template <typename Rl, typename StoreF>
__device__ __forceinline__ void env_to_freq(const LunaInst& I, Ws<Rl>& w, cpx<Rl>* x, StoreF&& store) {
    const int No = I.No, N = I.N, h = I.N / 2;
    cpx<Rl>* buf = w.main;
    cpx<Rl>* Z = block_fft<Rl, false>(x, w.main_alt ? ((x == buf) ? w.main_alt : buf) : nullptr, No, w.tw);
    for (int k = threadIdx.x; k < N; k += LUNA_BLOCK) {
        const int src = (k < h) ? k : (No - N + k);
        store(k, cvt<double>(Z[Swz<Rl>::f(src)]));
    }
    __syncthreads();
}

// envelope grid (EnvGrid): complex transforms with copy_scale_both! padding
template <typename Rl, typename LoadF, typename StoreF>
__device__ __forceinline__ void rhs_env(const LunaInst& I, Ws<Rl>& w, LoadF&& load, StoreF&& store) {
    int P;
    cpx<Rl>* x = env_to_time<Rl>(I, w, load, &P);
    // field scale; a taper's at this node is in outz[Nw]
    const double sc = I.grad ? I.outz[I.Nw].x : I.in_scale;
    pointwise_env<Rl>(I, w, x, P, sc);
    // with a pressure gradient the factor at the current z (outz, plain loads)
    env_to_freq<Rl>(I, w, x, [&](int k, cpx<double> X) {
        store(k, X * (I.grad ? reinterpret_cast<const cpx<double>*>(I.outz)[k]
                             : ldg(reinterpret_cast<const cpx<double>*>(I.outfac) + k)));
    });
}

template <typename Rl, typename LoadF, typename StoreF>
__device__ __forceinline__ void rhs(const LunaInst& I, Ws<Rl>& w, LoadF&& load, StoreF&& store) {
    if (I.kind == 0) rhs_real<Rl>(I, w, load, store);
    else rhs_env<Rl>(I, w, load, store);
}

// ------------------------------------------------------------------ stepfun filter
// Luna.jl:366-372: Eω .*= ωwin; Et = FT \ Eω; Et .*= twin; Eω = FT * Et (coarse grid),
// applied to yn after multiplying by exp(L*dz) (prop!_maybe, RK45.jl:225).
template <typename Rl>
__device__ __noinline__ void stepfun_filter(const LunaInst& I, Ws<Rl>& w, double2* yn, const double2* e1) {
    const int tid = threadIdx.x, T = LUNA_BLOCK;
    const int Nw = I.Nw, N = I.N;
    cpx<Rl>* buf = w.main;
    const cpx<double>* Y = reinterpret_cast<const cpx<double>*>(yn);
    const cpx<double>* P = reinterpret_cast<const cpx<double>*>(e1);
    auto ld = [&](int k) -> cpx<double> { return scale(__ldg(I.wwin + k), Y[k] * P[k]); };
    cpx<double>* Yo = reinterpret_cast<cpx<double>*>(yn);
    if (I.kind == 0) {
        const int M = N / 2;
        for (int k = tid; k <= M / 2; k += T) {
            const int km = M - k;
            cpx<double> Xk = (k < Nw) ? ld(k) : mk<double>(0, 0);
            cpx<double> Xm = (km == k) ? Xk : ((km < Nw) ? ld(km) : mk<double>(0, 0));
            if (k == 0) {
                Xk.y = 0;
                Xm.y = 0;
            }
            cpx<double> Wi = half_twiddle<Rl, true>(w.tw, k, M);
            cpx<double> Zk = (Xk + conj(Xm)) + mul_mi<double, true>(Wi * (Xk - conj(Xm)));
            buf[Swz<Rl>::f(k)] = cvt<Rl>(Zk);
            if (k != 0 && km != k) {
                cpx<double> Wmi = scale(-1.0, conj(Wi));
                cpx<double> Zm = (Xm + conj(Xk)) + mul_mi<double, true>(Wmi * (Xm - conj(Xk)));
                buf[Swz<Rl>::f(km)] = cvt<Rl>(Zm);
            }
        }
        __syncthreads();
        cpx<Rl>* x = block_fft<Rl, true>(buf, w.main_alt, M, w.tw);
        const int P = buf_split<Rl>(w.main_alt, M);
        const double inv = 1.0 / (double)N;
        for (int m = tid; m < M; m += T) {
            const int pos = Swz<Rl>::f(split_pos(m, M, P));
            cpx<Rl> e = x[pos];
            double a = (double)e.x * inv * __ldg(I.twin + 2 * m);
            double b = (double)e.y * inv * __ldg(I.twin + 2 * m + 1);
            x[pos] = mk<Rl>((Rl)a, (Rl)b);
        }
        __syncthreads();
        cpx<Rl>* Z = block_fft<Rl, false>(x, w.main_alt ? ((x == buf) ? w.main_alt : buf) : nullptr, M, w.tw);
        for (int k = tid; k < Nw; k += T) {
            const int km = (M - k) & (M - 1);
            cpx<double> Zk = cvt<double>(Z[Swz<Rl>::f(k & (M - 1))]);
            cpx<double> Zm = cvt<double>(Z[Swz<Rl>::f(km)]);
            cpx<double> X;
            if (k == 0) X = mk<double>(Zk.x + Zk.y, 0.0);
            else if (k == M) X = mk<double>(Zk.x - Zk.y, 0.0);
            else {
                cpx<double> Wk = half_twiddle<Rl, false>(w.tw, k, M);
                X = scale(0.5, Zk + conj(Zm)) + scale(0.5, mul_mi<double, false>(Wk * (Zk - conj(Zm))));
            }
            Yo[k] = X;
        }
    } else {
        for (int j = tid; j < N; j += T) buf[Swz<Rl>::f(j)] = cvt<Rl>(ld(j));
        __syncthreads();
        cpx<Rl>* x = block_fft<Rl, true>(buf, w.main_alt, N, w.tw);
        const int P = buf_split<Rl>(w.main_alt, N);
        const double inv = 1.0 / (double)N;
        for (int n = tid; n < N; n += T) {
            const int pos = Swz<Rl>::f(split_pos(n, N, P));
            x[pos] = cvt<Rl>(scale(inv * __ldg(I.twin + n), cvt<double>(x[pos])));
        }
        __syncthreads();
        cpx<Rl>* Z = block_fft<Rl, false>(x, w.main_alt ? ((x == buf) ? w.main_alt : buf) : nullptr, N, w.tw);
        for (int k = tid; k < N; k += T) Yo[k] = cvt<double>(Z[Swz<Rl>::f(k)]);
    }
    __syncthreads();
}

// ------------------------------------------------------------------ integrator
// Dormand-Prince tableau as shipped with the reference (dopri.jl:2-28): the step uses
// the 4th-order weights b5, error weights b5-b4 and the 4x7 dense-output matrix.
__device__ __constant__ double c_B[6][6] = {
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
__device__ __constant__ double c_nodes[6] = {1.0 / 5, 3.0 / 10, 4.0 / 5, 8.0 / 9, 1.0, 1.0};
__device__ __constant__ double c_b5[7] = {5179.0 / 57600, 0, 7571.0 / 16695, 393.0 / 640,
                                          -92097.0 / 339200, 187.0 / 2100, 1.0 / 40};
__device__ __constant__ double c_b4[7] = {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84, 0};
__device__ __constant__ double c_interp[4][7] = {
    {1, 0, 0, 0, 0, 0, 0},
    {-183.0 / 64, 0, 1500.0 / 371, -125.0 / 32, 9477.0 / 3392, -11.0 / 7, 3.0 / 2},
    {37.0 / 12, 0, -1000.0 / 159, 125.0 / 12, -729.0 / 106, 11.0 / 3, -4},
    {-145.0 / 128, 0, 1000.0 / 371, -375.0 / 64, 25515.0 / 6784, -55.0 / 28, 5.0 / 2}};

template <typename Kt> struct KT;
template <> struct KT<double> {
    static __device__ __forceinline__ cpx<double> ld(const void* p, int k) {
        return reinterpret_cast<const cpx<double>*>(p)[k];
    }
    static __device__ __forceinline__ void st(void* p, int k, cpx<double> v) {
        reinterpret_cast<cpx<double>*>(p)[k] = v;
    }
};
template <> struct KT<float> {
    static __device__ __forceinline__ cpx<double> ld(const void* p, int k) {
        return cvt<double>(reinterpret_cast<const cpx<float>*>(p)[k]);
    }
    static __device__ __forceinline__ void st(void* p, int k, cpx<double> v) {
        reinterpret_cast<cpx<float>*>(p)[k] = cvt<float>(v);
    }
};

// exp(L*d): FP64 throughout for the plain path; for the mixed path the phase is formed
// and reduced modulo 2*pi in FP64 and the trigonometry runs in FP32.
template <typename Rl>
__device__ __forceinline__ cpx<Rl> expLd(cpx<double> L, double d);
template <>
__device__ __forceinline__ cpx<double> expLd<double>(cpx<double> L, double d) {
    const double a = exp(L.x * d);
    double s, c;
    sincos(L.y * d, &s, &c);
    return mk<double>(a * c, a * s);
}
template <>
__device__ __forceinline__ cpx<float> expLd<float>(cpx<double> L, double d) {
    const double th = L.y * d;
    const double r = th - 6.283185307179586 * rint(th * 0.15915494309189535);
    float s, c;
    sincosf((float)r, &s, &c);
    const float a = expf((float)(L.x * d));
    return mk<float>(a * c, a * s);
}

template <typename Rl>
__device__ __forceinline__ cpx<double> inv_fac(cpx<Rl> f) {
    cpx<double> d = cvt<double>(f);
    const double inv = 1.0 / abs2(d);
    return scale(inv, conj(d));
}

// Dense output (RK45.jl:249-268) into row `out`; after an accepted step ks[1] holds k7,
// so the k1 and k7 coefficients both apply to that buffer. Bins r0, r0 + rs, r0 + 2 rs, ...
// (all bins by default; one residue class per CTA of a distributed instance).
template <typename Rl, typename Kt>
__device__ void interpolate_row(int Nw, const double2* linop, const Ctl& c, double ti, void* const* k,
                                const double2* py, const double2* pyn, double2* out, int r0 = 0, int rs = 1) {
    const cpx<double>* y = reinterpret_cast<const cpx<double>*>(py);
    const cpx<double>* yn = reinterpret_cast<const cpx<double>*>(pyn);
    const cpx<double>* L = reinterpret_cast<const cpx<double>*>(linop);
    cpx<double>* o = reinterpret_cast<cpx<double>*>(out);
    if (ti == c.t) {
        for (int i = r0 + rs * threadIdx.x; i < Nw; i += rs * LUNA_BLOCK) o[i] = y[i];
        return;
    }
    if (ti == c.tn) {
        for (int i = r0 + rs * threadIdx.x; i < Nw; i += rs * LUNA_BLOCK) o[i] = yn[i];
        return;
    }
    const double s = (ti - c.t) / c.dt;
    const double sp[4] = {s, s * s, s * s * s, (s * s) * (s * s)};
    double b[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        double acc = 0;
#pragma unroll
        for (int p = 0; p < 4; ++p) acc += sp[p] * c_interp[p][j];
        b[j] = acc;
    }
    const double d = ti - c.t;
    for (int i = r0 + rs * threadIdx.x; i < Nw; i += rs * LUNA_BLOCK) {
        cpx<double> yi = mk<double>(0, 0);
        cpx<double> k1 = KT<Kt>::ld(k[0], i);
        yi = yi + scale(b[0], k1);
#pragma unroll
        for (int j = 1; j < 6; ++j) yi = yi + scale(b[j], KT<Kt>::ld(k[j], i));
        yi = yi + scale(b[6], k1);
        cpx<double> v = y[i] + scale(c.dt, yi);
        o[i] = v * cvt<double>(expLd<double>(L[i], d));
    }
}

// ------------------------------------------------------------------ per-step statistics
// Block reductions returning the result in every thread (fixed order). `sh` holds at
// least 4 * LUNA_WARPS doubles; the calls end with a barrier, so `sh` can be reused.
__device__ __forceinline__ void block_argmax(double& v, int& i, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        if (v2 > v || (v2 == v && i2 < i)) {
            v = v2;
            i = i2;
        }
    }
    __syncthreads();
    if (lane == 0) {
        sh[wid] = v;
        sh[LUNA_WARPS + wid] = (double)i;
    }
    __syncthreads();
    v = sh[0];
    i = (int)sh[LUNA_WARPS];
    for (int q = 1; q < LUNA_WARPS; ++q) {
        const double v2 = sh[q];
        const int i2 = (int)sh[LUNA_WARPS + q];
        if (v2 > v || (v2 == v && i2 < i)) {
            v = v2;
            i = i2;
        }
    }
    __syncthreads();
}

// four index reductions at once: a, b by max; c, d by min
__device__ __forceinline__ void block_idx4(int& a, int& b, int& c, int& d, double* sh) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a = max(a, __shfl_xor_sync(0xffffffffu, a, o));
        b = max(b, __shfl_xor_sync(0xffffffffu, b, o));
        c = min(c, __shfl_xor_sync(0xffffffffu, c, o));
        d = min(d, __shfl_xor_sync(0xffffffffu, d, o));
    }
    __syncthreads();
    if (lane == 0) {
        sh[wid] = a;
        sh[LUNA_WARPS + wid] = b;
        sh[2 * LUNA_WARPS + wid] = c;
        sh[3 * LUNA_WARPS + wid] = d;
    }
    __syncthreads();
    for (int q = 0; q < LUNA_WARPS; ++q) {
        a = max(a, (int)sh[q]);
        b = max(b, (int)sh[LUNA_WARPS + q]);
        c = min(c, (int)sh[2 * LUNA_WARPS + q]);
        d = min(d, (int)sh[3 * LUNA_WARPS + q]);
    }
    __syncthreads();
}

__device__ __forceinline__ double linterpx(double x1, double x2, double y1, double y2, double val) {
    const double slope = (y2 - y1) / (x2 - x1);
    const double icpt = y1 - slope * x1;
    return (val - icpt) / slope;
}

// ------------------------------------------------------------------ pressure gradients
// Capillary.gradient (Capillary.jl:306-337) and LinearOps.make_linop (LinearOps.jl:337-360)
// evaluated at z. Every operation is an explicitly rounded IEEE operation (no contraction
// into fused multiply-adds) in the order of the host restatement: the group delay β1(z) is a
// finite difference with h = 1e-4 ω0, which turns one ulp of an effective index into ~1e-12
// of β1 and a visible time shift of the pulse, so host and device evaluate identical
// sequences.
__device__ __forceinline__ double grad_pressure(const LunaGrad* g, double z) {
    if (g->two_point) {
        if (z > g->Z[1]) return g->P[1];
        if (z <= 0) return g->P[0];
        return __dsqrt_rn(__dadd_rn(g->P2[0], __dmul_rn(__ddiv_rn(z, g->Z[1]), __dsub_rn(g->P2[1], g->P2[0]))));
    }
    const int n = g->npts;
    if (z <= g->Z[0]) return g->P[0];
    if (z >= g->Z[n - 1]) return g->P[n - 1];
    int i = 0;
    while (i + 1 < n - 1 && g->Z[i + 1] < z) ++i;  // last i with Z[i] < z
    const double f = __ddiv_rn(__dsub_rn(z, g->Z[i]), __dsub_rn(g->Z[i + 1], g->Z[i]));
    return __dsqrt_rn(__dadd_rn(g->P2[i], __dmul_rn(f, __dsub_rn(g->P2[i + 1], g->P2[i]))));
}

__device__ __forceinline__ double grad_density(const LunaGrad* g, double z) {
    const double p = grad_pressure(g, z);
    return __ddiv_rn(__dmul_rn(g->dens_a, p), __dadd_rn(1.0, __dmul_rn(g->dens_b, p)));
}

// core radius a(z): linear between nodes, the end values outside
__device__ __forceinline__ double grad_radius(const LunaGrad* g, double z) {
    const int n = g->nta;
    if (n == 1 || z <= g->ZA[0]) return g->A[0];
    if (z >= g->ZA[n - 1]) return g->A[n - 1];
    int i = 0;
    while (i + 1 < n - 1 && g->ZA[i + 1] < z) ++i;  // last i with ZA[i] < z
    const double f = __ddiv_rn(__dsub_rn(z, g->ZA[i]), __dsub_rn(g->ZA[i + 1], g->ZA[i]));
    return __dadd_rn(g->A[i], __dmul_rn(f, __dsub_rn(g->A[i + 1], g->A[i])));
}

__device__ __forceinline__ double grad_aeff(const LunaGrad* g, double a) {
    return __dmul_rn(__dmul_rn(a, a), g->aeff_intg);
}

// sqrt(coren^2 - nwg), coren = sqrt(1 + γ ρ), nwg = (unm/(k a))^2 (1 - i vn/(k a))^2 written
// as s^2 (p^2 - q^2, 2pq), p = 1 + Im vn/(k a), q = -Re vn/(k a); principal root from
// r = |w|, t = sqrt((r + |x|)/2): x >= 0 gives t + i y/(2t), else |y|/(2t) + i copysign(t, y)
__device__ __forceinline__ double2 grad_neff(double gam, double kc, double2 vn, double unm, double a, double rho,
                                             int loss) {
    const double ka = __dmul_rn(kc, a);
    const double s = __ddiv_rn(unm, ka);
    const double s2 = __dmul_rn(s, s);
    const double p = __dadd_rn(1.0, __ddiv_rn(vn.y, ka));
    const double q = -__ddiv_rn(vn.x, ka);
    const double nr = __dmul_rn(s2, __dsub_rn(__dmul_rn(p, p), __dmul_rn(q, q)));
    const double ni = __dmul_rn(s2, __dmul_rn(2.0, __dmul_rn(p, q)));
    const double cr = __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(gam, rho)));
    const double x = __dsub_rn(__dmul_rn(cr, cr), nr);
    const double y = -ni;
    const double r = __dsqrt_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
    double re, im;
    if (x >= 0) {
        const double t = __dsqrt_rn(__dmul_rn(__dadd_rn(r, x), 0.5));
        re = t;
        im = (t != 0) ? __ddiv_rn(y, __dmul_rn(2.0, t)) : 0.0;
    } else {
        const double t = __dsqrt_rn(__dmul_rn(__dsub_rn(r, x), 0.5));
        re = fabs(__ddiv_rn(y, __dmul_rn(2.0, t)));
        im = copysign(t, y);
    }
    return make_double2(re, loss ? im : 0.0);
}

// β1(z): 4-point central difference of x/c Re neff(x) (low-index rule) at ω0
__device__ __forceinline__ double grad_beta1(const LunaGrad* g, double rho, double a) {
    double f[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const double re = grad_neff(g->fd_gam[j], g->fd_xc[j], g->fd_vn[j], g->unm, a, rho, g->loss).x;
        f[j] = __dmul_rn(g->fd_xc[j], (re < 1e-3) ? 1e-3 : re);
    }
    const double num = __dadd_rn(__dsub_rn(__dadd_rn(-f[0], __dmul_rn(8.0, f[1])), __dmul_rn(8.0, f[2])), f[3]);
    return __ddiv_rn(num, g->fd_h12);
}

// The gradient/taper at z for the whole CTA: L(ω; z) into Lout (when wantL), the output
// factor ρ(z) sqrt(Aeff(z)) ofs/β(z) (ρ(z) ofs off sidx) into oout[0..Nw-1] and
// (field scale, Aeff) into oout[Nw]. One thread evaluates the scalars and passes them
// through bc (5 doubles of shared memory). On an envelope grid `om` holds ω - ω0 and,
// without THG, L gains + i β(ω0; z) (make_linop for EnvGrid, LinearOps.jl:363-388).
__device__ __noinline__ void grad_fill_to(const LunaInst& I, double* bc, double z, bool wantL, double2* Lout,
                                          double2* oout) {
    const LunaGrad* g = I.grad;
    __syncthreads();
    if (threadIdx.x == 0) {
        const double rho = grad_density(g, z);
        const double a = grad_radius(g, z);
        const double ae = grad_aeff(g, a);
        bc[0] = rho;
        bc[1] = a;
        bc[2] = wantL ? grad_beta1(g, rho, a) : 0.0;
        bc[3] = ae;
        double br = 0.0;
        if (wantL && g->bref) {
            // Modes.β(mode, ω0; z) = ω0/c Re neff(ω0; z), with the low-index rule of a taper
            const double re = grad_neff(g->ref_gam, g->ref_xc, g->ref_vn, g->unm, a, rho, g->loss).x;
            br = __dmul_rn(g->ref_xc, (g->nta > 1 && re < 1e-3) ? 1e-3 : re);
        }
        bc[4] = br;
        oout[I.Nw] = make_double2(g->in_base / sqrt(ae), ae);
    }
    __syncthreads();
    const double rho = bc[0], a = bc[1], b1 = bc[2], sae = sqrt(bc[3]), br = bc[4];
    const bool tapered = g->nta > 1;
    cpx<double>* Lz = reinterpret_cast<cpx<double>*>(Lout);
    cpx<double>* oz = reinterpret_cast<cpx<double>*>(oout);
    for (int i = threadIdx.x; i < I.Nw; i += LUNA_BLOCK) {
        const double wc = __ldg(g->wc + i);
        const double2 o = __ldg(g->ofs + i);
        if (wc == 0) {
            if (wantL) Lz[i] = mk<double>(0, 0);
            oz[i] = mk<double>(rho * o.x, rho * o.y);
            continue;
        }
        const double2 n = grad_neff(__ldg(g->gam + i), wc, __ldg(g->vn + i), g->unm, a, rho, g->loss);
        if (wantL) {
            const double re = fmax(n.x, 1e-3);                       // conj_clamp
            const double im = fmin(fmax(n.y, 0.0), __ldg(g->imcap + i));
            const double X = __dsub_rn(__dmul_rn(wc, re), __dmul_rn(__ldg(g->om + i), b1));
            Lz[i] = mk<double>(-__dmul_rn(wc, im), g->bref ? __dadd_rn(-X, br) : -X);
        }
        // β(z) = ω/c Re neff, with the low-index rule of neff(m, ω; z) for a taper
        const double nb = (tapered && n.x < 1e-3) ? 1e-3 : n.x;
        const double f = rho * sae / __dmul_rn(wc, nb);
        oz[i] = mk<double>(f * o.x, f * o.y);
    }
    __syncthreads();
}

// ... and, with wantH, the Raman spectrum at rho(z) of a density-dependent response (before
// a right-hand-side evaluation at z; grad_fill_to leaves rho in w.red[0])
template <typename Rl>
__device__ __forceinline__ void grad_fill(const LunaInst& I, Ws<Rl>& w, double z, bool wantL, bool wantH = true) {
    grad_fill_to(I, w.red, z, wantL, I.linz, I.outz);
    if (wantH && I.ramz) raman_h_at<Rl>(I, w, w.red[0]);
}

// Stats.default for a mode-averaged field-resolved transform (Stats.jl:495-532) on the
// accepted, window-filtered state Y at z with the next step dz, into row[LUNA_NSTATS]:
// z, dz, spectral centroid ω0 (Stats.jl:18-24), energy_ω (Fields.jl:510-520; SimpsonEven
// weights 17/48, 59/48, 43/48, 49/48 at both ends), peak power and peak intensity of the
// analytic field (plan_analytic, Stats.jl:434-462: 2*E[k] for k < Nw-1, inverse transform
// of length N), FWHM min/max with linear crossings (Maths.jl:128-190) and, with a plasma
// response, electron density and peak ionisation rate (Stats.jl:228-257).
template <typename Rl>
__device__ __noinline__ void step_stats(const LunaInst& I, Ws<Rl>& w, const double2* yn, double z, double dz,
                                        double* row) {
    const int tid = threadIdx.x, T = LUNA_BLOCK;
    const int Nw = I.Nw, N = I.N;
    const cpx<double>* Y = reinterpret_cast<const cpx<double>*>(yn);
    int ip = -1;
    for (int i = 0; i < I.nresp; ++i)
        if (I.resp[i].kind == LUNA_RESP_PLASMA_PPT || I.resp[i].kind == LUNA_RESP_PLASMA_ADK) ip = i;
    double sw = 0, s1 = 0, ss = 0;
    for (int k = tid; k < Nw; k += T) {
        const double a = abs2(Y[k]);
        s1 += a;
        sw += I.omega[k] * a;
        const int kk = min(k, Nw - 1 - k);
        const double wt = (kk == 0) ? 17.0 / 48 : (kk == 1) ? 59.0 / 48 : (kk == 2) ? 43.0 / 48 : (kk == 3) ? 49.0 / 48 : 1.0;
        ss += wt * a;
    }
    block_sum3(sw, s1, ss, w.red);
    __syncthreads();
    // analytic field
    cpx<Rl>* buf = w.main;
    for (int k = tid; k < N; k += T) buf[Swz<Rl>::f(k)] = (k < Nw - 1) ? cvt<Rl>(scale(2.0, Y[k])) : mk<Rl>(0, 0);
    __syncthreads();
    const cpx<Rl>* x = block_fft<Rl, true>(buf, w.main_alt, N, w.tw);
    const int P = buf_split<Rl>(w.main_alt, N);
    const double invN = 1.0 / (double)N;
    auto Pt = [&](int n) -> double { return abs2(scale(invN, cvt<double>(x[Swz<Rl>::f(split_pos(n, N, P))]))); };
    double vmax = -1.0;
    int imax = 0;
    double rs = 0, rmax = 0, redge = 0;
    // a taper's effective area and field scale at z
    const double aeff = I.grad ? grad_aeff(I.grad, grad_radius(I.grad, z)) : I.aeff;
    const double esc = I.grad ? 1.0 / sqrt(I.grad->eps0c2 * aeff) : I.escale;
    for (int n = tid; n < N; n += T) {
        const cpx<double> e = scale(invN, cvt<double>(x[Swz<Rl>::f(split_pos(n, N, P))]));
        const double pt = abs2(e);
        if (pt > vmax) {
            vmax = pt;
            imax = n;
        }
        if (ip >= 0) {
            const double E = e.x * esc;
            const double r = (double)eval_rate<Rl>(I.resp[ip], (Rl)fabs(E), w.flag);
            rs += r;
            rmax = fmax(rmax, r);
            if (n == 0 || n == N - 1) redge += r;
        }
    }
    block_argmax(vmax, imax, w.tot);
    {
        double c = 0;
        block_sum3(rs, redge, c, w.red);  // sum of the rates and r[0] + r[N-1]
        int dummy = 0;
        block_argmax(rmax, dummy, w.tot);
    }
    const double val = 0.5 * vmax;
    int minL = -1, maxR = -1, minR = N, maxL = N;
    for (int n = tid; n < N; n += T) {
        const double pt = Pt(n);
        if (n < imax && pt < val) minL = max(minL, n);
        if (n > imax && pt > val) maxR = max(maxR, n);
        if (n > imax && pt < val) minR = min(minR, n);
        if (n < imax && pt > val) maxL = min(maxL, n);
    }
    block_idx4(minL, maxR, minR, maxL, w.red);
    if (tid == 0) {
        const double* t = I.tgrid;
        double fmn = NAN, fmx = NAN;
        if (minL >= 0 && minR < N) {
            const double left = linterpx(t[minL], t[minL + 1], Pt(minL), Pt(minL + 1), val);
            const double right = linterpx(t[minR - 1], t[minR], Pt(minR - 1), Pt(minR), val);
            fmn = fabs(right - left);
        }
        if (maxL < N && maxR >= 0 && maxL >= 1 && maxR + 1 <= N - 1) {
            const double left = linterpx(t[maxL - 1], t[maxL], Pt(maxL - 1), Pt(maxL), val);
            const double right = linterpx(t[maxR], t[maxR + 1], Pt(maxR), Pt(maxR + 1), val);
            fmx = fabs(right - left);
        }
        const double h = I.omega[1] - I.omega[0];
        const double wl = I.omega[Nw - 1];
        row[0] = z;
        row[1] = dz;
        row[2] = sw / s1;
        row[3] = 2.0 * 3.141592653589793 / (wl * wl) * (h * ss);
        row[4] = vmax;
        row[5] = vmax / aeff;
        row[6] = fmn;
        row[7] = fmx;
        if (ip >= 0) {
            const double dtg = t[1] - t[0];
            const double Tr = dtg * (rs - 0.5 * redge);  // trapezoid integral of the rate
            const double rho = I.grad ? grad_density(I.grad, z) : 1.0;  // coef is 1 then
            row[8] = (1.0 - exp(-Tr)) * I.resp[ip].coef * rho;
            row[9] = rmax;
        } else {
            row[8] = NAN;
            row[9] = NAN;
        }
    }
    __syncthreads();
}

// Weak error norm, PI step control, step limits and step bookkeeping after the stage
// evaluations (RK45.jl:167-192, 343-354, 374-406); one thread. sy, syn and se are the
// sums of |y|^2, |yn|^2 and |yerr|^2; flags are the status bits raised by the RHS.
__device__ __forceinline__ void control_step(LunaInst& I, Ctl& c, double sy, double syn, double se, int flags,
                                             bool writer = true) {
    const double errwt = fmax(fmax(sqrt(sy), sqrt(syn)), I.atol);
    const double err = sqrt(se) / I.rtol / errwt;
    c.err = err;
    int ok = err <= 1.0;
    // stepcontrolPI! (RK45.jl:374-396)
    const double b1 = 3.0 / 5 / 5, b2 = -1.0 / 5 / 5, eps = 0.8;
    if (ok) {
        if (c.errlast == 0) c.errlast = err;
        double fac = (err == 0) ? 1.5 : I.safety * pow(eps / err, b1) * pow(eps / c.errlast, b2);
        c.dtn = fac * c.dt;
        c.errlast = err;
    } else {
        if (!isfinite(err)) c.dtn = c.dt / 2;
        else c.dtn = c.dt * fmax(0.1, I.safety * pow(err, -1.0 / 5));
    }
    // steplims! (RK45.jl:399-406)
    if (c.dtn > I.max_dt) c.dtn = I.max_dt;
    else if (c.dtn < I.min_dt) {
        c.dtn = I.min_dt;
        ok = 1;
    }
    // replay mode: follow a given step sequence (dt of the next step, accept flag)
    if (I.replay && c.steps < I.nreplay) {
        ok = I.replay[2 * c.steps + 1] != 0.0;
        if (c.steps + 1 < I.nreplay) c.dtn = I.replay[2 * (c.steps + 1)];
    }
    c.ok = ok;
    if (ok) c.tn = c.t + c.dt;
    c.steps += 1;
    const long long si = c.steps - 1;
    if (writer && I.steplog && si < I.steplog_cap) {
        I.steplog[4 * si + 0] = c.t;
        I.steplog[4 * si + 1] = c.dt;
        I.steplog[4 * si + 2] = err;
        I.steplog[4 * si + 3] = (double)ok;
    }
    if (ok) {
        c.repeated = 0;
        if (writer) I.accepted += 1;
    } else {
        c.repeated += 1;
        if (writer) I.rejected += 1;
        if (c.repeated > I.repeat_limit) {
            c.status = ST_REPEAT_LIMIT;
            c.done = 1;
        }
    }
    if (flags & (1 << ST_FIELD_ABOVE_EMAX)) {
        c.status = ST_FIELD_ABOVE_EMAX;
        c.done = 1;
    }
    if (flags & (1 << ST_WAIT_TIMEOUT)) {
        c.status = ST_WAIT_TIMEOUT;
        c.done = 1;
    }
    if (I.max_steps > 0 && c.steps >= I.max_steps && !c.done) {
        c.status = ST_STEP_BUDGET;
        c.done = 1;
    }
}

template <typename Rl, typename Kt>
__device__ void solve_instance(LunaInst& I, Ws<Rl>& w, Ctl& c) {
    const int tid = threadIdx.x, T = LUNA_BLOCK;
    const int Nw = I.Nw;
    // constant linop, or L(z) of the current stage node (pressure gradient)
    const cpx<double>* L = reinterpret_cast<const cpx<double>*>(I.grad ? I.linz : I.linop);
    void** k = c.k;
    if (tid == 0)
        for (int j = 0; j < 7; ++j) k[j] = I.k[j];
    cpx<double>* e1 = reinterpret_cast<cpx<double>*>(I.e1);
    double2* py = I.y;
    double2* pyn = I.yn;
    long long nrhs = 0;
    if (tid == 0) {
        c.t = c.tn = I.z0;
        c.dt = c.dtn = I.dz0;
        c.err = c.errlast = 0;
        c.ok = 0;
        c.done = 0;
        c.status = 0;
        c.repeated = 0;
        c.steps = 0;
        *w.flag = 0;
    }
    // y = yn = y0
    {
        const cpx<double>* y0 = reinterpret_cast<const cpx<double>*>(I.y0);
        cpx<double>* y = reinterpret_cast<cpx<double>*>(py);
        cpx<double>* yn = reinterpret_cast<cpx<double>*>(pyn);
        for (int i = tid; i < Nw; i += T) {
            y[i] = y0[i];
            yn[i] = y0[i];
        }
    }
    __syncthreads();
    // k1 = fbar(y0, t, t): propagation by exp(L*0) == 1
    if (I.grad) grad_fill<Rl>(I, w, I.z0, false);
    {
        const cpx<double>* y = reinterpret_cast<const cpx<double>*>(py);
        void* k0 = k[0];
        rhs<Rl>(I, w, [&](int i) { return y[i]; }, [&](int i, cpx<double> v) { KT<Kt>::st(k0, i, v); });
        ++nrhs;
    }
    int saved = 0;
    bool swap_y = false;  // y <- yn at the next step start (after an accepted step)
    while (true) {
        __syncthreads();
        if (!(c.tn <= I.zmax) || c.done) break;
        // ---------------- evaluate! (RK45.jl:209-223)
        if (swap_y) {
            double2* tmp = py;
            py = pyn;
            pyn = tmp;
        }
        const double dprop = c.tn - c.t;  // k1 <- exp(L*(tn-t)) k1
        __syncthreads();
        if (tid == 0) {
            c.dt = c.dtn;
            c.t = c.tn;
        }
        __syncthreads();
        const double t0 = c.t, dt = c.dt;
        const cpx<double>* y = reinterpret_cast<const cpx<double>*>(py);
        for (int s = 0; s < 6; ++s) {
            // stage node t + c_s dt and the propagation distance to it, rounded as written
            const double zs = __dadd_rn(t0, __dmul_rn(c_nodes[s], dt));
            const double d = __dsub_rn(zs, t0);
            const bool reuse = (s == 5);  // nodes 5 and 6 coincide
            if (!reuse) {
                if (I.grad) grad_fill<Rl>(I, w, zs, true);
                for (int i = tid; i < Nw; i += T) {
                    cpx<Rl> f = expLd<Rl>(L[i], d);
                    w.efac[i] = f;
                    if (s == 4) e1[i] = cvt<double>(f);
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
                return cvt<double>(w.efac[i]) * acc;
            };
            auto store = [&](int i, cpx<double> v) { KT<Kt>::st(kout, i, v * inv_fac<Rl>(w.efac[i])); };
            rhs<Rl>(I, w, load, store);
            ++nrhs;
        }
        // ---------------- step! (RK45.jl:167-192): combine, weak norm, PI control
        double sy = 0, syn = 0, se = 0;
        {
            cpx<double>* yn = reinterpret_cast<cpx<double>*>(pyn);
            double cb5[7], cer[7];
#pragma unroll
            for (int j = 0; j < 7; ++j) {
                cb5[j] = dt * c_b5[j];
                cer[j] = c_b5[j] - c_b4[j];
            }
            for (int i = tid; i < Nw; i += T) {
                cpx<double> yi = y[i];
                cpx<double> acc = yi;
                cpx<double> er = mk<double>(0, 0);
#pragma unroll
                for (int j = 0; j < 7; ++j) {
                    cpx<double> kj = KT<Kt>::ld(k[j], i);
                    if (c_b5[j] != 0) acc = acc + scale(cb5[j], kj);
                    if (cer[j] != 0) er = er + scale(cer[j], scale(dt, kj));
                }
                yn[i] = acc;
                sy += abs2(yi);
                syn += abs2(acc);
                se += abs2(er);
            }
        }
        block_sum3(sy, syn, se, w.red);
        if (tid == 0) control_step(I, c, sy, syn, se, *w.flag);
        __syncthreads();
        if (c.done && c.status != 0) break;
        if (c.ok) {
            // FSAL: ks[1] <- ks[7]
            __syncthreads();
            if (tid == 0) {
                void* tmp = k[0];
                k[0] = k[6];
                k[6] = tmp;
            }
            __syncthreads();
            // prop!_maybe + stepfun window filter on yn
            stepfun_filter<Rl>(I, w, pyn, I.e1);
            // Stats.default of the filtered state (MemoryOutput calls it before the saves)
            if (I.stats && I.nstats < I.stats_cap) {
                step_stats<Rl>(I, w, pyn, c.tn, c.dtn, I.stats + (size_t)LUNA_NSTATS * I.nstats);
                if (tid == 0) I.nstats += 1;
            }
            // GridCondition saves (Output.jl:65-82, 490-502)
            while (saved < I.saveN && I.zsave[saved] <= c.tn) {
                // make_prop! evaluates a z-dependent linop at the save point itself
                if (I.grad) grad_fill<Rl>(I, w, I.zsave[saved], true, false);
                interpolate_row<Rl, Kt>(Nw, I.grad ? I.linz : I.linop, c, I.zsave[saved], k, py, pyn,
                                        I.saves + (size_t)saved * Nw);
                ++saved;
            }
            swap_y = true;
        } else {
            // yn = y; prop!_maybe with tn == t multiplies by exp(0) == 1
            cpx<double>* yn = reinterpret_cast<cpx<double>*>(pyn);
            for (int i = tid; i < Nw; i += T) yn[i] = y[i];
            swap_y = false;
        }
    }
    __syncthreads();
    if (tid == 0) {
        // final state: the last accepted yn (already filtered)
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
    __syncthreads();
}

}  // namespace luna
