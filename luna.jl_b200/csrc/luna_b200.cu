// Kernels and the C ABI of libluna_b200 (see include/luna_b200.h).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstddef>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/luna_b200.h"
#include "dist.cuh"
#include "modal.cuh"
#include "tc_gemm.cuh"

using namespace luna;

// ===================================================================== kernels

// Persistent solver: each CTA pulls instances from `counter` until the list is empty and
// integrates each one to completion (RK45.solve loop, RK45.jl:43-78).
// With `list`, the q-th instance pulled is insts[list[q]] (q < n), else insts[q].
template <typename Rl, typename Kt>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
solve_kernel(LunaInst* insts, int n, int* counter, TwTab<Rl> tw, int smem_bytes, const int* list) {
    extern __shared__ __align__(256) char smem[];
    __shared__ Ctl ctl;
    __shared__ int sidx;
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) sidx = atomicAdd(counter, 1);
        __syncthreads();
        const int q = sidx;
        if (q >= n) break;
        LunaInst& I = insts[list ? list[q] : q];
        if (threadIdx.x == 0) {
            unsigned long long t;
            unsigned int sm;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
            I.t_begin = t;
            I.sm = (int)sm;
        }
        Ws<Rl> w;
        plan_ws<Rl>(I, smem, smem_bytes, w, tw);
        solve_instance<Rl, Kt>(I, w, ctl);
        if (threadIdx.x == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            I.t_end = t;
        }
    }
}

// ---------------------------------------------------------------- Raman clusters
// Helper CTA (rank 1 or 2) of a Raman cluster. The Raman convolution of an instance with
// No time samples is a 2*No-point real convolution, i.e. an Mr = No point complex
// transform of the packed input z[m] = (E[2m]^2, E[2m+1]^2), m < No/2 (zero above), and
// only P[m < No/2] is used. With HM = Mr/2 the even and odd frequencies separate:
//   Z[2j]   = FFT_HM(z)[j],               Z[2j+1] = FFT_HM(z[m] e^{-2 pi i m/Mr})[j],
//   P[m]    = IFFT_HM(Z'_even)[m] + e^{+2 pi i m/Mr} IFFT_HM(Z'_odd)[m],
// and the real-transform split / response product / split of the convolution pairs k
// with Mr-k, which has the parity of k. Each helper therefore holds one half (HM points)
// in its own shared memory; rank 0 adds the two halves (distributed shared memory).
template <typename Rl>
__device__ void cluster_helper(LunaInst* insts, char* smem, int smem_bytes, const TwTab<Rl>& tw, unsigned rank,
                               ClBox* box, int* err) {
    namespace cg = cooperative_groups;
    const int tid = threadIdx.x, T = LUNA_BLOCK;
    cpx<Rl>* buf = reinterpret_cast<cpx<Rl>*>(smem + LUNA_SMALL_BYTES);
    __shared__ int s_ok;
    int seen = 0;
    const int par = (int)rank - 1;
    while (true) {
        if (tid == 0) {
            const long long t0 = clock64();
            int ok = 1;
            while ((int)cl_ld_acquire(&box->seq) == seen) {
                if (clock64() - t0 > CL_WAIT_CYCLES) {
                    ok = 0;
                    break;
                }
            }
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) {
            if (tid == 0) atomicOr(err, 1);
            return;
        }
        seen = box->seq;
        if (box->cmd != CL_RAMAN) return;  // CL_EXIT
        const LunaInst& I = insts[box->inst];
        if (rank == 3) {
            // plasma helper: rho * P_plasma of every sample into this CTA's buffer
            int ip = -1;
            for (int i = 0; i < I.nresp; ++i)
                if (I.resp[i].kind == LUNA_RESP_PLASMA_PPT || I.resp[i].kind == LUNA_RESP_PLASMA_ADK) ip = i;
            Ws<Rl> w;
            plan_ws<Rl>(I, smem, smem_bytes, w, tw, nullptr, true);
            if (tid == 0) *w.flag = 0;
            __syncthreads();
            if (ip >= 0) {
                const cpx<Rl>* xr = cooperative_groups::this_cluster().map_shared_rank(
                    reinterpret_cast<cpx<Rl>*>(__cvta_shared_to_generic(box->xaddr)), 0);
                plasma_only<Rl>(I, w, xr, w.main, box->M, box->P, (double)box->sc, ip);
            }
            __syncthreads();
            if (tid == 0) {
                cl_st(cl_map(&box->pflag, 0), (unsigned)*w.flag);
                cl_fence();
                cl_st_release(cl_map(&box->done[2], 0), (unsigned)seen);
            }
            continue;
        }
        const LunaResp* rr = nullptr;
        for (int i = 0; i < I.nresp; ++i)
            if (I.resp[i].kind == LUNA_RESP_RAMAN) rr = &I.resp[i];
        const int Mr = I.No, HM = Mr / 2;
        const int M = box->M, P = box->P;
        const Rl sc = (Rl)box->sc;
        const int Ph = fft_nsplit<Rl>(HM);
        const unsigned tsh = TW_LOG_MMAX - ilog2i((unsigned)Mr);
        const cpx<Rl>* xr = cg::this_cluster().map_shared_rank(
            reinterpret_cast<cpx<Rl>*>(__cvta_shared_to_generic(box->xaddr)), 0);
        // packed squares of the field (odd half: times e^{-2 pi i m/Mr}), split order
        // (four remote loads in flight per thread)
        for (int m0 = tid; m0 < HM; m0 += 4 * T) {
            cpx<Rl> e[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int m = m0 + q * T;
                e[q] = (m < HM) ? xr[Swz<Rl>::f(split_pos(m, M, P))] : mk<Rl>(0, 0);
            }
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int m = m0 + q * T;
                if (m >= HM) continue;
                const Rl e0 = e[q].x * sc, e1 = e[q].y * sc;
                cpx<Rl> v = mk<Rl>(e0 * e0, e1 * e1);
                if (par) v = v * twiddle<Rl, false>(tw, (unsigned)m << tsh);
                buf[Swz<Rl>::f(split_pos(m, HM, Ph))] = v;
            }
        }
        __syncthreads();
        cpx<Rl>* Z = block_fft<Rl, false>(buf, nullptr, HM, tw);
        const cpx<Rl>* H = reinterpret_cast<const cpx<Rl>*>(rr->H);
        // real-transform split, response product, inverse split (as in raman_conv) for the
        // frequencies k = 2t + par <= Mr/2 and their partners Mr - k
        for (int t = tid;; t += T) {
            const int k = 2 * t + par;
            if (k > Mr / 2) break;
            const int km = (Mr - k) & (Mr - 1);
            const int jk = k >> 1, jm = km >> 1;
            cpx<double> Zk = cvt<double>(Z[Swz<Rl>::f(jk)]);
            cpx<double> Zm = cvt<double>(Z[Swz<Rl>::f(jm)]);
            cpx<double> Wk = half_twiddle<Rl, false>(tw, k, Mr);
            cpx<double> a = Zk + conj(Zm), b = Zk - conj(Zm);
            cpx<double> Xk = scale(0.5, a) + scale(0.5, mul_mi<double, false>(Wk * b));
            cpx<double> Xm;
            if (k == 0) {
                Xk = mk<double>(Zk.x + Zk.y, 0.0);
                Xm = mk<double>(Zk.x - Zk.y, 0.0);
            } else {
                cpx<double> Wm = scale(-1.0, conj(Wk));
                cpx<double> a2 = Zm + conj(Zk), b2 = Zm - conj(Zk);
                Xm = scale(0.5, a2) + scale(0.5, mul_mi<double, false>(Wm * b2));
            }
            cpx<double> Yk = Xk * cvt<double>(ldg(H + k));
            cpx<double> Ym = Xm * cvt<double>(ldg(H + (Mr - k)));
            cpx<double> Wi = conj(Wk);
            cpx<double> Zk2 = (Yk + conj(Ym)) + mul_mi<double, true>(Wi * (Yk - conj(Ym)));
            Z[Swz<Rl>::f(jk)] = cvt<Rl>(Zk2);
            if (k != 0 && km != k) {
                cpx<double> Wmi = scale(-1.0, Wk);
                cpx<double> Zm2 = (Ym + conj(Yk)) + mul_mi<double, true>(Wmi * (Ym - conj(Yk)));
                Z[Swz<Rl>::f(jm)] = cvt<Rl>(Zm2);
            }
        }
        __syncthreads();
        cpx<Rl>* Y = block_fft<Rl, true>(Z, nullptr, HM, tw);
        if (par) {
            for (int m = tid; m < HM; m += T) {
                const int pos = Swz<Rl>::f(split_pos(m, HM, Ph));
                Y[pos] = Y[pos] * twiddle<Rl, true>(tw, (unsigned)m << tsh);
            }
        }
        __syncthreads();
        if (tid == 0) {
            cl_fence();
            cl_st_release(cl_map(&box->done[par], 0), (unsigned)seen);
        }
    }
}

// Persistent solver with Raman clusters (launched with clusters of 3 CTAs). Phase 1: each
// cluster integrates the instances of `big` (FP32 Raman buffers too large for one CTA's
// shared memory), rank 0 running the solver and ranks 1-2 the Raman halves. Phase 2: once
// `big` is empty, every CTA integrates instances of `reg` on its own (no cluster traffic).
template <typename Rl, typename Kt>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
solve_kernel_cl(LunaInst* insts, const int* big, int nbig, int* big_counter, const int* reg, int nreg,
                int* reg_counter, TwTab<Rl> tw, int smem_bytes, int* err) {
    namespace cg = cooperative_groups;
    extern __shared__ __align__(256) char smem[];
    __shared__ Ctl ctl;
    __shared__ ClBox box;
    __shared__ int sidx;
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    if (threadIdx.x == 0) {
        box.seq = 0;
        box.cmd = 0;
        for (int h = 0; h < CL_HELPERS; ++h) box.done[h] = 0;
        box.pflag = 0;
        box.inst = -1;
    }
    cl.sync();  // every mailbox is initialised before any remote write
    if (rank == 0) {
        while (true) {
            __syncthreads();
            if (threadIdx.x == 0) sidx = (box.cmd == -1) ? nbig : atomicAdd(big_counter, 1);
            __syncthreads();
            const int q = sidx;
            if (q >= nbig) break;
            const int i = big[q];
            LunaInst& I = insts[i];
            if (threadIdx.x == 0) {
                unsigned long long t;
                unsigned int sm;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
                I.t_begin = t;
                I.sm = (int)sm;
                box.inst = i;
            }
            __syncthreads();
            Ws<Rl> w;
            plan_ws<Rl>(I, smem, smem_bytes, w, tw, nullptr, true);
            w.cl = &box;
            w.rem_e = cl.map_shared_rank(reinterpret_cast<cpx<Rl>*>(smem + LUNA_SMALL_BYTES), 1);
            w.rem_o = cl.map_shared_rank(reinterpret_cast<cpx<Rl>*>(smem + LUNA_SMALL_BYTES), 2);
            w.rem_p = cl.map_shared_rank(reinterpret_cast<cpx<Rl>*>(smem + LUNA_SMALL_BYTES), 3);
            solve_instance<Rl, Kt>(I, w, ctl);
            if (threadIdx.x == 0) {
                unsigned long long t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                I.t_end = t;
            }
        }
        // release the helpers (not after a timeout: they may have left already)
        if (threadIdx.x == 0 && box.cmd != -1) {
            const int seq = ++box.seq;
            for (unsigned h = 1; h <= CL_HELPERS; ++h) cl_st(cl_map(&box.cmd, h), CL_EXIT);
            cl_fence();
            for (unsigned h = 1; h <= CL_HELPERS; ++h) cl_st_release(cl_map(&box.seq, h), (unsigned)seq);
        }
        __syncthreads();
    } else if (rank <= CL_HELPERS) {
        cluster_helper<Rl>(insts, smem, smem_bytes, tw, rank, &box, err);
    }
    __syncthreads();
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) sidx = atomicAdd(reg_counter, 1);
        __syncthreads();
        const int q = sidx;
        if (q >= nreg) break;
        LunaInst& I = insts[reg[q]];
        if (threadIdx.x == 0) {
            unsigned long long t;
            unsigned int sm;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
            I.t_begin = t;
            I.sm = (int)sm;
        }
        Ws<Rl> w;
        plan_ws<Rl>(I, smem, smem_bytes, w, tw);
        solve_instance<Rl, Kt>(I, w, ctl);
        if (threadIdx.x == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            I.t_end = t;
        }
    }
}

// Persistent solver on clusters of R CTAs. Phase 1: each cluster integrates the
// instances of `dl` (the long ones, in priority order) together, every CTA holding one
// residue class of the frequency bins and one block of the time samples. Phase 2: once
// `dl` is empty, every CTA integrates instances of `reg` on its own.
template <typename Rl, typename Kt, int R>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
solve_kernel_dist(LunaInst* insts, const int* dl, int nd, int* d_counter, const int* reg, int nreg,
                  int* reg_counter, TwTab<Rl> tw, int smem_bytes) {
    namespace cg = cooperative_groups;
    extern __shared__ __align__(256) char smem[];
    __shared__ Ctl ctl;
    __shared__ int sidx;
    cg::cluster_group cl = cg::this_cluster();
    const int rank = (int)cl.block_rank();
    while (true) {
        if (rank == 0 && threadIdx.x == 0) sidx = atomicAdd(d_counter, 1);
        cl.sync();
        const int q = *cl.map_shared_rank(&sidx, 0);
        cl.sync();  // rank 0's index is read everywhere before the next pull overwrites it
        if (q >= nd) break;
        LunaInst& I = insts[dl[q]];
        if (rank == 0 && threadIdx.x == 0) {
            unsigned long long t;
            unsigned int sm;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
            I.t_begin = t;
            I.sm = (int)sm;
        }
        DWs<Rl> d;
        plan_dws<Rl, R>(I, smem, d, tw, rank);
        solve_instance_dist<Rl, Kt, R>(I, d, ctl);
        if (rank == 0 && threadIdx.x == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            I.t_end = t;
        }
    }
    while (true) {
        __syncthreads();
        if (threadIdx.x == 0) sidx = atomicAdd(reg_counter, 1);
        __syncthreads();
        const int q = sidx;
        if (q >= nreg) break;
        LunaInst& I = insts[reg[q]];
        if (threadIdx.x == 0) {
            unsigned long long t;
            unsigned int sm;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            asm volatile("mov.u32 %0, %%smid;" : "=r"(sm));
            I.t_begin = t;
            I.sm = (int)sm;
        }
        Ws<Rl> w;
        plan_ws<Rl>(I, smem, smem_bytes, w, tw);
        solve_instance<Rl, Kt>(I, w, ctl);
        if (threadIdx.x == 0) {
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            I.t_end = t;
        }
    }
}

// One right-hand-side evaluation nl = T(Eω) on one CTA (TransModeAvg call).
template <typename Rl>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
rhs_kernel(LunaInst* inst, const double2* Ew, double2* nl, TwTab<Rl> tw, int smem_bytes, int* status, double z) {
    extern __shared__ __align__(256) char smem[];
    LunaInst& I = *inst;
    Ws<Rl> w;
    plan_ws<Rl>(I, smem, smem_bytes, w, tw);
    if (threadIdx.x == 0) *w.flag = 0;
    __syncthreads();
    if (I.grad) grad_fill<Rl>(I, w, z, false);  // ρ(z) and the normalisation at z
    const cpx<double>* E = reinterpret_cast<const cpx<double>*>(Ew);
    cpx<double>* o = reinterpret_cast<cpx<double>*>(nl);
    rhs<Rl>(I, w, [&](int k) { return E[k]; }, [&](int k, cpx<double> v) { o[k] = v; });
    __syncthreads();
    if (threadIdx.x == 0) *status = (*w.flag & (1 << ST_FIELD_ABOVE_EMAX)) ? ST_FIELD_ABOVE_EMAX : ST_OK;
}

// linop!(out, z) of a pressure-gradient plan and the output factor at z, on one CTA.
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
grad_linop_kernel(LunaInst I, double z, double2* L, double2* of) {
    __shared__ double bc[5];
    grad_fill_to(I, bc, z, true, L, of);
}

// Raman response spectrum at plan creation (Raman.jl:256-262, Nonlinear.jl:306-307):
// h(t) = w(t) * sum_c hpre_c(t) exp(-t/tau2_c) on the first half of a 2*No grid,
// H[k] = rfft(hscale * h)[k], k = 0..No, computed in FP64. The response is normalised by
// hscale = 1/max|hpre| so that its spectrum is representable in FP32 (molecular responses
// are ~1e-48 in SI units); the plan folds max|hpre| * hdt / (2*No) into the FP64 coefficient.
template <typename Rl>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
raman_h_kernel(LunaResp r, int No, double hscale, cpx<double>* buf, cpx<Rl>* H, TwTab<double> tw) {
    const int tid = threadIdx.x;
    const int P = fft_nsplit<double>(No);
    for (int m = tid; m < No; m += LUNA_BLOCK) {
        double a = 0, b = 0;
        if (m < No / 2) {
            a = raman_sample(r, No, 2 * m, r.tau2, hscale);
            b = raman_sample(r, No, 2 * m + 1, r.tau2, hscale);
        }
        buf[Swz<double>::f(split_pos(m, No, P))] = mk<double>(a, b);
    }
    __syncthreads();
    cpx<double>* Z = block_fft<double, false>(buf, nullptr, No, tw);
    const int M = No;
    for (int k = tid; k <= M; k += LUNA_BLOCK) {
        const int kk = k & (M - 1);
        const int km = (M - k) & (M - 1);
        cpx<double> Zk = Z[Swz<double>::f(kk)];
        cpx<double> Zm = Z[Swz<double>::f(km)];
        cpx<double> X;
        if (k == 0) X = mk<double>(Zk.x + Zk.y, 0.0);
        else if (k == M) X = mk<double>(Zk.x - Zk.y, 0.0);
        else {
            cpx<double> Wk = half_twiddle<double, false>(tw, k, M);
            X = scale(0.5, Zk + conj(Zm)) + scale(0.5, mul_mi<double, false>(Wk * (Zk - conj(Zm))));
        }
        H[k] = cvt<Rl>(X);
    }
}

// ===================================================================== host side
namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return fail(LUNA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

struct TwDev {
    TwTab<double> d;
    TwTab<float> f;
};

std::mutex g_tw_mu;
std::map<int, TwDev> g_tw;

int get_tw(TwDev& out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_tw_mu);
    auto it = g_tw.find(dev);
    if (it != g_tw.end()) {
        out = it->second;
        return LUNA_OK;
    }
    std::vector<cpx<double>> lo(TW_NLO), hi(TW_NHI);
    std::vector<cpx<float>> lof(TW_NLO), hif(TW_NHI);
    const double two_pi = 6.283185307179586476925286766559;
    for (int j = 0; j < TW_NLO; ++j) {
        double a = -two_pi * (double)j / (double)TW_MMAX;
        lo[j] = mk<double>(std::cos(a), std::sin(a));
        lof[j] = mk<float>((float)lo[j].x, (float)lo[j].y);
    }
    for (int j = 0; j < TW_NHI; ++j) {
        double a = -two_pi * (double)(j * TW_NLO) / (double)TW_MMAX;
        hi[j] = mk<double>(std::cos(a), std::sin(a));
        hif[j] = mk<float>((float)hi[j].x, (float)hi[j].y);
    }
    TwDev t;
    void* p;
    CK(cudaMalloc(&p, sizeof(cpx<double>) * (TW_NLO + TW_NHI)));
    CK(cudaMemcpy(p, lo.data(), sizeof(cpx<double>) * TW_NLO, cudaMemcpyHostToDevice));
    CK(cudaMemcpy((char*)p + sizeof(cpx<double>) * TW_NLO, hi.data(), sizeof(cpx<double>) * TW_NHI,
                  cudaMemcpyHostToDevice));
    t.d.lo = (const cpx<double>*)p;
    t.d.hi = (const cpx<double>*)((char*)p + sizeof(cpx<double>) * TW_NLO);
    CK(cudaMalloc(&p, sizeof(cpx<float>) * (TW_NLO + TW_NHI)));
    CK(cudaMemcpy(p, lof.data(), sizeof(cpx<float>) * TW_NLO, cudaMemcpyHostToDevice));
    CK(cudaMemcpy((char*)p + sizeof(cpx<float>) * TW_NLO, hif.data(), sizeof(cpx<float>) * TW_NHI,
                  cudaMemcpyHostToDevice));
    t.f.lo = (const cpx<float>*)p;
    t.f.hi = (const cpx<float>*)((char*)p + sizeof(cpx<float>) * TW_NLO);
    g_tw[dev] = t;
    out = t;
    return LUNA_OK;
}

bool is_pow2(int x) { return x > 0 && (x & (x - 1)) == 0; }

int max_smem_optin() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    return v - 1024;  // leave room for the kernels' static shared memory
}

template <typename Rl>
size_t smem_wanted(const LunaInst& I) {
    const size_t c = sizeof(cpx<Rl>);
    size_t s = LUNA_SMALL_BYTES;
    s += align_up((size_t)main_len(I) * c, 256);
    if (needs_hilbert(I)) s += align_up((size_t)(I.No / 2) * c, 256);
    s += align_up((size_t)I.Nw * c, 256);
    if (has_raman(I)) s += align_up((size_t)I.No * c, 256);
    return s;
}

}  // namespace

struct luna_plan {
    int precision = 0;
    LunaInst proto{};
    std::vector<void*> allocs;
    bool has_raman = false;
    void* d_hbuf = nullptr;      // FP64 work buffer of the Raman spectrum build ([No] complex)
    LunaGrad* d_grad = nullptr;  // pressure gradient (device copy), or null
    // single-call RHS resources
    bool inst_stale = false;     // d_inst predates a change of proto
    double2* d_outz = nullptr;   // output factor at z (pressure gradient)
    LunaInst* d_inst = nullptr;
    void* d_gscr = nullptr;
    double2* d_Ew = nullptr;
    double2* d_nl = nullptr;
    int* d_status = nullptr;
    cudaStream_t stream = nullptr;
};

struct luna_batch {
    int n = 0;
    int precision = 0;
    std::vector<luna_plan*> plans;
    luna_solve_opts opts{};
    std::vector<LunaInst> h;
    LunaInst* d_insts = nullptr;
    int* d_counter = nullptr;
    // Raman clusters (mixed precision): instances whose FP32 Raman buffer does not fit in
    // one CTA's shared memory run on clusters of 3 CTAs; the rest in cost order
    int nbig = 0, nreg = 0, cl_grid = 0;
    int* d_big = nullptr;
    int* d_reg = nullptr;
    int* d_cl_counters = nullptr;  // [0] big, [1] regular, [2] error flag
    std::vector<int> big, reg;     // host copies of the two lists
    std::vector<void*> allocs;
    std::vector<double2*> y0buf;  // per instance y (holds y0 before the run)
    std::vector<double2*> ybuf, ynbuf;
    std::vector<double*> steplogs;
    std::vector<double*> zsave_own;  // per-instance save points (optional)
    double* d_zsave = nullptr;
    int smem = 0;
    int grid = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t stream2 = nullptr;  // single-CTA solver beside the cluster solver
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, evf = nullptr, evj = nullptr;
    int reg_grid = 0;
    // distributed instances (clusters of DIST_R CTAs per instance, DIST_R_BIG for the
    // longest ones, each on its own stream)
    int ndist = 0, dist_grid = 0, ncl_max = 0, nsm = 0;
    int* d_dist = nullptr;
    std::vector<int> dist, elig;
    int ndist16 = 0, dist16_grid = 0, ncl16_max = 0;
    int* d_dist16 = nullptr;
    std::vector<int> dist16, elig16;
    cudaStream_t stream3 = nullptr;
    cudaEvent_t evj3 = nullptr;
    std::vector<int> shape;  // per instance: 0 the work-estimate rule, 1 one CTA, 2 a cluster,
                             // 3 a cluster of DIST_R_BIG
};

namespace {

template <typename T>
int dalloc(std::vector<void*>& allocs, T** p, size_t bytes) {
    void* q = nullptr;
    CK(cudaMalloc(&q, bytes > 0 ? bytes : 16));
    allocs.push_back(q);
    *p = reinterpret_cast<T*>(q);
    return LUNA_OK;
}

template <typename T>
int upload(std::vector<void*>& allocs, const T* src, size_t n, const T** dst) {
    T* p = nullptr;
    int rc = dalloc(allocs, &p, n * sizeof(T));
    if (rc) return rc;
    CK(cudaMemcpy(p, src, n * sizeof(T), cudaMemcpyHostToDevice));
    *dst = p;
    return LUNA_OK;
}

void free_all(std::vector<void*>& allocs) {
    for (void* p : allocs) cudaFree(p);
    allocs.clear();
}

// Which instances of a batch run distributed, from per-instance work estimates: the eligible
// ones whose estimate is at least the mean load of an SM (total / SMs), i.e. the long poles
// of the batch (a cluster costs more SM time than one CTA; shorter Raman instances whose
// buffers overflow one CTA run single with them in global memory). Every SM that can hold a
// cluster starts as one (longest instances first); the single-CTA instances fill the SMs
// left over and the clusters once their list is empty. Both lists in priority order.
int dist_partition(luna_batch* b, const double* pr) {
    const int n = b->n;
    double W = 0;
    for (int i = 0; i < n; ++i) W += pr[i];
    const double thr = W / std::max(1, b->nsm);
    // 0: one CTA, 1: a cluster of DIST_R, 2: a cluster of DIST_R_BIG. The big clusters take
    // the eligible instances whose estimate is at least four times the mean SM load (those
    // that would set the makespan even on a cluster of DIST_R)
    std::vector<char> isd(n, 0), big(n, 0);
    for (int i = 0; i < n; ++i) big[i] = 0;
    for (int i : b->elig16) big[i] = 1;
    for (int i : b->elig) {
        const int sh = b->shape.empty() ? 0 : b->shape[i];
        isd[i] = sh == 2 || sh == 3 || (sh == 0 && pr[i] >= thr);
        if (isd[i] && big[i] && b->ncl16_max > 0 && (sh == 3 || (sh == 0 && pr[i] >= 4.0 * thr))) isd[i] = 2;
    }
    b->dist.clear();
    b->dist16.clear();
    b->reg.clear();
    for (int i = 0; i < n; ++i) (isd[i] == 2 ? b->dist16 : isd[i] ? b->dist : b->reg).push_back(i);
    auto by = [&](int a, int c) { return pr[a] > pr[c]; };
    std::stable_sort(b->dist.begin(), b->dist.end(), by);
    std::stable_sort(b->dist16.begin(), b->dist16.end(), by);
    std::stable_sort(b->reg.begin(), b->reg.end(), by);
    b->ndist = (int)b->dist.size();
    b->ndist16 = (int)b->dist16.size();
    b->nreg = (int)b->reg.size();
    const int n16 = std::min(b->ncl16_max, b->ndist16);
    // a big cluster takes the room of DIST_R_BIG / DIST_R small ones
    const int ncl = std::min(std::max(1, b->ncl_max - n16 * (DIST_R_BIG / DIST_R)), b->ndist);
    b->dist16_grid = DIST_R_BIG * n16;
    b->dist_grid = (b->ndist > 0) ? DIST_R * ncl : 0;
    b->reg_grid = std::max(0, std::min(b->nreg, b->nsm - b->dist_grid - b->dist16_grid));
    if (b->ndist > 0) CK(cudaMemcpy(b->d_dist, b->dist.data(), sizeof(int) * b->ndist, cudaMemcpyHostToDevice));
    if (b->ndist16 > 0) CK(cudaMemcpy(b->d_dist16, b->dist16.data(), sizeof(int) * b->ndist16, cudaMemcpyHostToDevice));
    if (b->nreg > 0) CK(cudaMemcpy(b->d_reg, b->reg.data(), sizeof(int) * b->nreg, cudaMemcpyHostToDevice));
    return LUNA_OK;
}

// Distributed instances of a batch: the long ones (No >= dist_min_no, default 16384) that
// the cluster solver supports, each on DIST_R CTAs, in the batch's precision (FP32 or FP64
// sub-transforms and responses). Sets b->elig and the partition when at least one cluster
// fits on the device; a batch without eligible instances is left unchanged.
template <typename Rl>
int dist_setup(luna_batch* b, const luna_solve_opts* opts, int nsm) {
    const int n = b->n;
    const int maxs = max_smem_optin();
    const size_t cs = sizeof(cpx<Rl>);
    std::vector<int> dl, dl16;
    std::vector<double> cost(n);
    size_t dsm = 0;
    const int dmin = opts->dist_min_no > 0 ? opts->dist_min_no : 16384;
    auto fits = [&](const LunaInst& I, int R) {
        const int M = I.No / 2, Mc = I.N / 2;
        return M % R == 0 && M / R >= 2 * LUNA_BLOCK && M / R <= FftEmax<Rl>::v * LUNA_BLOCK && Mc % R == 0 &&
               Mc / R >= 64 && Mc <= M && I.Nw <= Mc + 1 && dist_smem_bytes(I.No, cs, R) <= (size_t)maxs;
    };
    for (int i = 0; i < n; ++i) {
        const LunaInst& I = b->h[i];
        const bool ok = I.kind == 0 && !I.grad && !needs_hilbert(I) && opts->stats_cap <= 0 && I.No >= dmin &&
                        fits(I, DIST_R);
        if (ok) {
            dl.push_back(i);
            dsm = std::max(dsm, dist_smem_bytes(I.No, cs));
            if (fits(I, DIST_R_BIG)) dl16.push_back(i);
        }
        cost[i] = (double)I.No * std::log2((double)I.No) * (has_raman(I) ? 2.0 : 1.0);
    }
    if (dl.empty()) return LUNA_OK;
    const int sm = (int)std::max<size_t>((size_t)b->smem, dsm);
    if (cudaFuncSetAttribute(solve_kernel_dist<Rl, Rl, DIST_R>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess ||
        cudaFuncSetAttribute(solve_kernel<Rl, Rl>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) != cudaSuccess)
        return fail(LUNA_ERR_CUDA, "batch_create: cannot set shared memory size (distributed solver)");
    auto max_clusters = [&](auto kern, int R) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = R;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(R * 32, 1, 1);
        cfg.blockDim = dim3(LUNA_BLOCK, 1, 1);
        cfg.dynamicSmemBytes = sm;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int ncl = 0;
        if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) != cudaSuccess) {
            cudaGetLastError();
            ncl = 0;
        }
        return ncl;
    };
    const int ncl = max_clusters(solve_kernel_dist<Rl, Rl, DIST_R>, DIST_R);
    if (ncl < 1) return LUNA_OK;
    int ncl16 = 0;
    if (!dl16.empty() &&
        cudaFuncSetAttribute(solve_kernel_dist<Rl, Rl, DIST_R_BIG>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm) == cudaSuccess &&
        cudaFuncSetAttribute(solve_kernel_dist<Rl, Rl, DIST_R_BIG>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess)
        ncl16 = max_clusters(solve_kernel_dist<Rl, Rl, DIST_R_BIG>, DIST_R_BIG);
    cudaGetLastError();
    b->smem = sm;
    b->elig = dl;
    b->elig16 = ncl16 > 0 ? dl16 : std::vector<int>();
    b->ncl_max = ncl;
    b->ncl16_max = ncl16;
    b->nsm = nsm;
    if (dalloc(b->allocs, &b->d_dist, sizeof(int) * n) || dalloc(b->allocs, &b->d_dist16, sizeof(int) * n) ||
        dalloc(b->allocs, &b->d_reg, sizeof(int) * n) || dalloc(b->allocs, &b->d_cl_counters, 4 * sizeof(int)))
        return LUNA_ERR_CUDA;
    return dist_partition(b, cost.data());
}

// The distributed solvers on their clusters (DIST_R_BIG on a third stream, DIST_R) and the
// single-CTA solver on the SMs left over (second stream), all in the batch's precision;
// every kernel takes single-CTA instances once its own list is empty.
template <typename Rl>
int dist_launch(luna_batch* b, const TwTab<Rl>& tw) {
    int* c = b->d_cl_counters;  // [0] clusters, [1] single CTAs, [2] error flag, [3] big clusters
    auto cfg_for = [&](int R, int grid, cudaStream_t st, cudaLaunchAttribute* at) {
        cudaLaunchConfig_t cfg = {};
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = R;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(grid, 1, 1);
        cfg.blockDim = dim3(LUNA_BLOCK, 1, 1);
        cfg.dynamicSmemBytes = b->smem;
        cfg.stream = st;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        return cfg;
    };
    CK(cudaEventRecord(b->evf, b->stream));
    if (b->reg_grid > 0) CK(cudaStreamWaitEvent(b->stream2, b->evf, 0));
    if (b->dist16_grid > 0) {
        CK(cudaStreamWaitEvent(b->stream3, b->evf, 0));
        cudaLaunchAttribute at16[1];
        cudaLaunchConfig_t cfg16 = cfg_for(DIST_R_BIG, b->dist16_grid, b->stream3, at16);
        CK(cudaLaunchKernelEx(&cfg16, solve_kernel_dist<Rl, Rl, DIST_R_BIG>, b->d_insts, (const int*)b->d_dist16,
                              b->ndist16, c + 3, (const int*)b->d_reg, b->nreg, c + 1, tw, b->smem));
        CK(cudaEventRecord(b->evj3, b->stream3));
    }
    if (b->dist_grid > 0) {
        cudaLaunchAttribute at[1];
        cudaLaunchConfig_t cfg = cfg_for(DIST_R, b->dist_grid, b->stream, at);
        CK(cudaLaunchKernelEx(&cfg, solve_kernel_dist<Rl, Rl, DIST_R>, b->d_insts, (const int*)b->d_dist, b->ndist, c,
                              (const int*)b->d_reg, b->nreg, c + 1, tw, b->smem));
    }
    if (b->dist16_grid > 0) CK(cudaStreamWaitEvent(b->stream, b->evj3, 0));
    if (b->reg_grid > 0) {
        solve_kernel<Rl, Rl><<<b->reg_grid, LUNA_BLOCK, b->smem, b->stream2>>>(b->d_insts, b->nreg, c + 1, tw, b->smem,
                                                                              (const int*)b->d_reg);
        CK(cudaEventRecord(b->evj, b->stream2));
        CK(cudaStreamWaitEvent(b->stream, b->evj, 0));
    }
    return LUNA_OK;
}

}  // namespace

extern "C" {

const char* luna_b200_last_error(void) { return g_err.c_str(); }

int luna_b200_version(void) { return 1; }

int luna_b200_plan_create(const luna_grid_desc* g, const luna_resp_desc* resps, int nresp, int precision,
                          luna_plan** out) {
    if (!g || !out || nresp < 0 || nresp > LUNA_MAX_RESP || (nresp > 0 && !resps))
        return fail(LUNA_ERR_BAD_ARG, "plan_create: null argument or too many responses");
    if (precision != LUNA_PREC_FP64 && precision != LUNA_PREC_MIXED)
        return fail(LUNA_ERR_BAD_ARG, "plan_create: unknown precision");
    if (g->kind != 0 && g->kind != 1) return fail(LUNA_ERR_BAD_ARG, "plan_create: grid kind must be 0 or 1");
    if (!is_pow2(g->N) || !is_pow2(g->No) || g->No < g->N || g->N < 16)
        return fail(LUNA_ERR_BAD_ARG, "plan_create: N and No must be powers of two with 16 <= N <= No");
    if (g->kind == 0 && g->Nw != g->N / 2 + 1)
        return fail(LUNA_ERR_BAD_ARG, "plan_create: RealGrid needs Nw == N/2 + 1");
    if (g->kind == 1 && g->Nw != g->N) return fail(LUNA_ERR_BAD_ARG, "plan_create: EnvGrid needs Nw == N");
    if (2 * g->No > TW_MMAX) return fail(LUNA_ERR_UNSUPPORTED, "plan_create: No too large");
    {
        // every transform must fit one CTA's split transform (8 sub-transforms)
        const int Mmain = (g->kind == 0) ? g->No / 2 : g->No;
        const int lim = (precision == LUNA_PREC_FP64) ? FftMmax<double>::v : FftMmax<float>::v;
        bool raman = false;
        for (int i = 0; i < nresp; ++i)
            raman = raman || resps[i].kind == LUNA_RESP_RAMAN || resps[i].kind == LUNA_RESP_RAMAN_NOTHG;
        if (Mmain > lim || (raman && g->No > lim) || g->No > FftMmax<double>::v * 2)
            return fail(LUNA_ERR_UNSUPPORTED, "plan_create: grid too large for one CTA");
        if (g->No < 2 * LUNA_BLOCK)
            return fail(LUNA_ERR_UNSUPPORTED, "plan_create: oversampled grid below 1024 samples");
    }
    if (!g->outfac || !g->wwin || !g->towin || !g->twin) return fail(LUNA_ERR_BAD_ARG, "plan_create: null grid array");
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
        return fail(LUNA_ERR_CUDA, "plan_create: no CUDA device available");
    TwDev tw;
    int rc = get_tw(tw);
    if (rc) return rc;

    luna_plan* p = new luna_plan();
    p->precision = precision;
    LunaInst& I = p->proto;
    memset(&I, 0, sizeof(I));
    I.kind = g->kind;
    I.N = g->N;
    I.Nw = g->Nw;
    I.No = g->No;
    I.in_scale = g->in_scale;
#define UP(src, n, dst)                                          \
    do {                                                         \
        int rc_ = upload(p->allocs, (src), (size_t)(n), (dst));  \
        if (rc_) {                                               \
            free_all(p->allocs);                                 \
            delete p;                                            \
            return rc_;                                          \
        }                                                        \
    } while (0)
    const double* tmp;
    UP(g->outfac, 2 * (size_t)g->Nw, &tmp);
    I.outfac = (const double2*)tmp;
    UP(g->wwin, g->Nw, &I.wwin);
    UP(g->towin, g->No, &I.towin);
    UP(g->twin, g->N, &I.twin);
    if (g->omega && g->t) {
        UP(g->omega, g->Nw, &I.omega);
        UP(g->t, g->N, &I.tgrid);
    }
    I.aeff = g->aeff;
    I.escale = g->escale;
    I.nresp = nresp;
    int nplasma = 0, nraman = 0;
    for (int i = 0; i < nresp; ++i) {
        const luna_resp_desc& d = resps[i];
        LunaResp& r = I.resp[i];
        memset(&r, 0, sizeof(r));
        r.kind = d.kind;
        r.coef = d.coef;
        switch (d.kind) {
            case LUNA_RESP_KERR_FIELD_NOTHG:
                r.kind = LUNA_RESP_KERR_FIELD;
                r.hilb = 1;
                // fall through
            case LUNA_RESP_KERR_FIELD:
                if (g->kind != 0) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "Kerr_field needs a RealGrid"); }
                break;
            case LUNA_RESP_KERR_ENV_THG:
                if (!d.cthg) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "Kerr_env_thg needs its exp(2iω0t) table"); }
                if (g->kind == 1) {
                    const double* c;
                    UP(d.cthg, 2 * (size_t)g->No, &c);
                    r.cthg = reinterpret_cast<const double2*>(c);
                }
                r.kind = LUNA_RESP_KERR_ENV;
                // fall through
            case LUNA_RESP_KERR_ENV:
                if (g->kind != 1) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "Kerr_env needs an EnvGrid"); }
                break;
            case LUNA_RESP_PLASMA_PPT:
            case LUNA_RESP_PLASMA_ADK: {
                if (g->kind != 0) { free_all(p->allocs); delete p; return fail(LUNA_ERR_UNSUPPORTED, "plasma response for envelope fields is not implemented (as in the reference)"); }
                if (!(d.preionfrac >= 0.0 && d.preionfrac <= 1.0)) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "preionfrac must be between 0 and 1"); }
                if (++nplasma > 1) { free_all(p->allocs); delete p; return fail(LUNA_ERR_UNSUPPORTED, "at most one plasma response"); }
                r.ionpot = d.ionpot;
                r.dt = d.dt;
                r.preion = d.preionfrac;
                r.eratio = d.eratio;
                if (d.kind == LUNA_RESP_PLASMA_PPT) {
                    if (d.spl_n < 4 || !d.spl_x || !d.spl_y || !d.spl_D) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "PPT spline table missing"); }
                    UP(d.spl_x, d.spl_n, &r.sx);
                    UP(d.spl_y, d.spl_n, &r.sy);
                    UP(d.spl_D, d.spl_n, &r.sD);
                    std::vector<float> fx(d.spl_n), fy(d.spl_n), fD(d.spl_n);
                    for (int j = 0; j < d.spl_n; ++j) {
                        fx[j] = (float)d.spl_x[j];
                        fy[j] = (float)d.spl_y[j];
                        fD[j] = (float)d.spl_D[j];
                    }
                    UP(fx.data(), d.spl_n, &r.sxf);
                    UP(fy.data(), d.spl_n, &r.syf);
                    UP(fD.data(), d.spl_n, &r.sDf);
                    r.sn = d.spl_n;
                    r.Emin = d.spl_x[0];
                    r.Emax = d.spl_x[d.spl_n - 1];
                } else {
                    r.adk_pre = d.adk_pre;
                    r.adk_a = d.adk_a;
                    r.adk_b = d.adk_b;
                    r.adk_pw = d.adk_pw;
                    r.adk_thr = d.adk_thr;
                }
                break;
            }
            case LUNA_RESP_RAMAN_NOTHG:
            case LUNA_RESP_RAMAN: {
                if (d.kind == LUNA_RESP_RAMAN_NOTHG) {
                    if (g->kind != 0) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "RamanPolarField(thg=false) needs a RealGrid"); }
                    r.kind = LUNA_RESP_RAMAN;
                    r.hilb = 1;
                }
                p->has_raman = true;
                if (++nraman > 1) { free_all(p->allocs); delete p; return fail(LUNA_ERR_UNSUPPORTED, "at most one Raman response"); }
                if (d.ncomp < 1 || !d.hpre || !d.tau2 || !d.hwin || !d.htt) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "Raman response tables missing"); }
                r.ncomp = d.ncomp;
                r.hdt = d.hdt;
                double hmax = 0;
                for (size_t j = 0; j < (size_t)d.ncomp * g->No; ++j) hmax = std::max(hmax, std::fabs(d.hpre[j]));
                if (!(hmax > 0)) hmax = 1;
                r.coef = d.coef * hmax * d.hdt / (2.0 * (double)g->No);
                UP(d.hpre, (size_t)d.ncomp * g->No, &r.hpre);
                UP(d.tau2, d.ncomp, &r.tau2);
                UP(d.hwin, g->No, &r.hwin);
                UP(d.htt, g->No, &r.htt);
                r.hscale = 1.0 / hmax;
                if (d.tau2_rho) {
                    // density laws of the dephasing times (used once a gradient is attached)
                    bool dep = false;
                    for (int c = 0; c < d.ncomp; ++c) {
                        const double m = d.tau2_rho[4 * c];
                        if (m != 0.0 && m != 1.0 && m != 2.0) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "Raman tau2_rho: unknown model"); }
                        dep = dep || m != 0.0;
                    }
                    if (dep) {
                        if (d.ncomp > LUNA_RAMAN_MAXC || !(d.amg > 0)) { free_all(p->allocs); delete p; return fail(LUNA_ERR_BAD_ARG, "Raman tau2_rho: at most 4 components and amg > 0"); }
                        UP(d.tau2_rho, 4 * (size_t)d.ncomp, &r.t2rho);
                        r.amg = d.amg;
                    }
                }
                // spectrum of the response, computed once on the device in FP64
                cpx<double>* b1 = nullptr;
                if (dalloc(p->allocs, &b1, sizeof(cpx<double>) * g->No)) {
                    free_all(p->allocs); delete p; return LUNA_ERR_CUDA;
                }
                p->d_hbuf = b1;
                if (precision == LUNA_PREC_FP64) {
                    cpx<double>* H = nullptr;
                    if (dalloc(p->allocs, &H, sizeof(cpx<double>) * (g->No + 1))) { free_all(p->allocs); delete p; return LUNA_ERR_CUDA; }
                    raman_h_kernel<double><<<1, LUNA_BLOCK>>>(r, g->No, 1.0 / hmax, b1, H, tw.d);
                    r.H = H;
                } else {
                    cpx<float>* H = nullptr;
                    if (dalloc(p->allocs, &H, sizeof(cpx<float>) * (g->No + 1))) { free_all(p->allocs); delete p; return LUNA_ERR_CUDA; }
                    raman_h_kernel<float><<<1, LUNA_BLOCK>>>(r, g->No, 1.0 / hmax, b1, H, tw.d);
                    r.H = H;
                }
                cudaError_t e = cudaDeviceSynchronize();
                if (e == cudaSuccess) e = cudaGetLastError();
                if (e != cudaSuccess) { free_all(p->allocs); delete p; return fail(LUNA_ERR_CUDA, std::string("raman_h_kernel: ") + cudaGetErrorString(e)); }
                break;
            }
            default:
                free_all(p->allocs);
                delete p;
                return fail(LUNA_ERR_UNSUPPORTED, "unknown response kind");
        }
    }
#undef UP
    *out = p;
    return LUNA_OK;
}

void luna_b200_plan_destroy(luna_plan* p) {
    if (!p) return;
    if (p->stream) cudaStreamDestroy(p->stream);
    free_all(p->allocs);
    delete p;
}

static int launch_rhs(luna_plan* p, const double2* Ew, double2* nl, cudaStream_t st, double z) {
    TwDev tw;
    int rc = get_tw(tw);
    if (rc) return rc;
    if (!p->d_inst || p->inst_stale) {
        LunaInst I = p->proto;
        if (!p->d_gscr) {
            size_t gb = (p->precision == LUNA_PREC_FP64) ? gscr_bytes<double>(I) : gscr_bytes<float>(I);
            if (dalloc(p->allocs, &p->d_gscr, gb)) return LUNA_ERR_CUDA;
        }
        I.gscr = p->d_gscr;
        if (I.grad) {
            if (!p->d_outz && dalloc(p->allocs, &p->d_outz, sizeof(double2) * (I.Nw + 1))) return LUNA_ERR_CUDA;
            I.outz = p->d_outz;
        }
        if (!p->d_inst && dalloc(p->allocs, &p->d_inst, sizeof(LunaInst))) return LUNA_ERR_CUDA;
        CK(cudaMemcpy(p->d_inst, &I, sizeof(LunaInst), cudaMemcpyHostToDevice));
        if (!p->d_status && dalloc(p->allocs, &p->d_status, sizeof(int))) return LUNA_ERR_CUDA;
        p->inst_stale = false;
    }
    const int maxs = max_smem_optin();
    if (p->precision == LUNA_PREC_FP64) {
        int sm = (int)std::min<size_t>(smem_wanted<double>(p->proto), (size_t)maxs);
        CK(cudaFuncSetAttribute(rhs_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        rhs_kernel<double><<<1, LUNA_BLOCK, sm, st>>>(p->d_inst, Ew, nl, tw.d, sm, p->d_status, z);
    } else {
        int sm = (int)std::min<size_t>(smem_wanted<float>(p->proto), (size_t)maxs);
        CK(cudaFuncSetAttribute(rhs_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        rhs_kernel<float><<<1, LUNA_BLOCK, sm, st>>>(p->d_inst, Ew, nl, tw.f, sm, p->d_status, z);
    }
    CK(cudaGetLastError());
    return LUNA_OK;
}

int luna_b200_plan_set_gradient(luna_plan* p, const luna_gradient_desc* g) {
    if (!p) return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: null plan");
    if (!g) {
        p->proto.grad = nullptr;
        p->inst_stale = true;
        if (p->proto.ramz) {
            // back to the spectrum at the dephasing times given at plan creation
            LunaResp& r = p->proto.resp[p->proto.ramz - 1];
            r.hz = 0;
            p->proto.ramz = 0;
            TwDev tw;
            int rc = get_tw(tw);
            if (rc) return rc;
            if (p->precision == LUNA_PREC_FP64)
                raman_h_kernel<double><<<1, LUNA_BLOCK>>>(r, p->proto.No, r.hscale, (cpx<double>*)p->d_hbuf, (cpx<double>*)const_cast<void*>(r.H), tw.d);
            else
                raman_h_kernel<float><<<1, LUNA_BLOCK>>>(r, p->proto.No, r.hscale, (cpx<double>*)p->d_hbuf, (cpx<float>*)const_cast<void*>(r.H), tw.d);
            CK(cudaGetLastError());
            CK(cudaDeviceSynchronize());
        }
        return LUNA_OK;
    }
    if (p->proto.kind == 1 && g->env_ref != 0 && g->env_ref != 1)
        return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: env_ref must be 0 or 1");
    if (g->npts < 2 || g->npts > LUNA_GRAD_MAXPTS) return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: npts out of range");
    if (g->two_point && g->npts != 2) return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: a two-point fill has npts == 2");
    for (int i = 0; i + 1 < g->npts; ++i)
        if (!(g->Z[i + 1] > g->Z[i])) return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: Z must increase");
    if (g->two_point && g->Z[0] != 0.0) return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: a two-point fill starts at z = 0");
    for (int i = 0; i < g->npts; ++i)
        if (!(g->P[i] >= 0) || g->P2[i] != g->P[i] * g->P[i])
            return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: pressures must be >= 0 with P2 = P*P");
    if (g->nta < 1 || g->nta > LUNA_GRAD_MAXPTS) return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: nta out of range");
    for (int i = 0; i < g->nta; ++i)
        if (!(g->A[i] > 0) || (i + 1 < g->nta && !(g->ZA[i + 1] > g->ZA[i])))
            return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: radii must be positive at increasing ZA");
    if (!(g->unm > 0) || !(g->aeff_intg > 0) || !(g->in_base > 0) || !(g->eps0c2 > 0))
        return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: mode constants must be positive");
    if (!g->gam || !g->vn || !g->wc || !g->om || !g->imcap || !g->ofs || !(g->fd_h12 > 0))
        return fail(LUNA_ERR_BAD_ARG, "plan_set_gradient: null table");
    const size_t Nw = (size_t)p->proto.Nw;
    LunaGrad h;
    memset(&h, 0, sizeof(h));
    h.npts = g->npts;
    h.two_point = g->two_point;
    h.loss = g->loss;
    for (int i = 0; i < g->npts; ++i) {
        h.Z[i] = g->Z[i];
        h.P[i] = g->P[i];
        h.P2[i] = g->P2[i];
    }
    h.dens_a = g->dens_a;
    h.dens_b = g->dens_b;
    h.nta = g->nta;
    for (int i = 0; i < g->nta; ++i) {
        h.ZA[i] = g->ZA[i];
        h.A[i] = g->A[i];
    }
    h.unm = g->unm;
    h.aeff_intg = g->aeff_intg;
    h.in_base = g->in_base;
    h.eps0c2 = g->eps0c2;
    for (int j = 0; j < 4; ++j) {
        h.fd_xc[j] = g->fd_xc[j];
        h.fd_gam[j] = g->fd_gam[j];
        h.fd_vn[j] = make_double2(g->fd_vn[2 * j], g->fd_vn[2 * j + 1]);
    }
    h.fd_h12 = g->fd_h12;
    // envelope grids without THG: the reference propagation constant β(ω0; z) is taken out
    h.bref = (p->proto.kind == 1) ? g->env_ref : 0;
    h.ref_xc = g->ref_xc;
    h.ref_gam = g->ref_gam;
    h.ref_vn = make_double2(g->ref_vn[0], g->ref_vn[1]);
    const double* t;
    if (upload(p->allocs, g->gam, Nw, &h.gam) || upload(p->allocs, g->vn, 2 * Nw, &t)) return LUNA_ERR_CUDA;
    h.vn = (const double2*)t;
    if (upload(p->allocs, g->wc, Nw, &h.wc) || upload(p->allocs, g->om, Nw, &h.om) ||
        upload(p->allocs, g->imcap, Nw, &h.imcap) || upload(p->allocs, g->ofs, 2 * Nw, &t))
        return LUNA_ERR_CUDA;
    h.ofs = (const double2*)t;
    const LunaGrad* d = nullptr;
    if (upload(p->allocs, &h, 1, &d)) return LUNA_ERR_CUDA;
    // a Raman response with density-dependent dephasing: its spectrum (the plan's own
    // buffer for the RHS entry points; batches give every instance one) is rebuilt at ρ(z)
    for (int i = 0; i < p->proto.nresp; ++i) {
        LunaResp& r = p->proto.resp[i];
        if (r.kind == LUNA_RESP_RAMAN && r.t2rho) {
            r.hz = 1;
            p->proto.ramz = i + 1;
        }
    }
    p->d_grad = const_cast<LunaGrad*>(d);
    p->proto.grad = p->d_grad;
    p->inst_stale = true;
    return LUNA_OK;
}

int luna_b200_plan_linop(luna_plan* p, double z, double* linop, double* outfac) {
    if (!p || !linop) return fail(LUNA_ERR_BAD_ARG, "plan_linop: null argument");
    if (!p->proto.grad) return fail(LUNA_ERR_BAD_ARG, "plan_linop: the plan has no pressure gradient");
    const size_t bytes = sizeof(double2) * p->proto.Nw;
    double2 *dL = nullptr, *dO = nullptr;
    CK(cudaMalloc(&dL, 2 * bytes + sizeof(double2)));
    dO = dL + p->proto.Nw;
    grad_linop_kernel<<<1, LUNA_BLOCK>>>(p->proto, z, dL, dO);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(linop, dL, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && outfac) e = cudaMemcpy(outfac, dO, bytes, cudaMemcpyDeviceToHost);
    cudaFree(dL);
    if (e != cudaSuccess) return fail(LUNA_ERR_CUDA, std::string("plan_linop: ") + cudaGetErrorString(e));
    return LUNA_OK;
}

int luna_b200_rhs_device(luna_plan* p, double* nl_dev, const double* Ew_dev, double z, void* stream) {
    if (!p || !nl_dev || !Ew_dev) return fail(LUNA_ERR_BAD_ARG, "rhs_device: null argument");
    return launch_rhs(p, (const double2*)Ew_dev, (double2*)nl_dev, (cudaStream_t)stream, z);
}

int luna_b200_rhs(luna_plan* p, double* nl, const double* Ew, double z) {
    if (!p || !nl || !Ew) return fail(LUNA_ERR_BAD_ARG, "rhs: null argument");
    const size_t bytes = sizeof(double2) * p->proto.Nw;
    if (!p->d_Ew) {
        if (dalloc(p->allocs, &p->d_Ew, bytes) || dalloc(p->allocs, &p->d_nl, bytes)) return LUNA_ERR_CUDA;
        CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    }
    CK(cudaMemcpyAsync(p->d_Ew, Ew, bytes, cudaMemcpyHostToDevice, p->stream));
    int rc = launch_rhs(p, p->d_Ew, p->d_nl, p->stream, z);
    if (rc) return rc;
    int st = 0;
    CK(cudaMemcpyAsync(nl, p->d_nl, bytes, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaMemcpyAsync(&st, p->d_status, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    if (st == ST_FIELD_ABOVE_EMAX) return fail(LUNA_FIELD_ABOVE_EMAX, "Field strength exceeds maximum for PPT ionisation rate.");
    return LUNA_OK;
}

// ---------------------------------------------------------------- batches
int luna_b200_batch_create(luna_plan* const* plans, int n, const luna_solve_opts* opts, luna_batch** out) {
    if (!plans || n <= 0 || !opts || !out) return fail(LUNA_ERR_BAD_ARG, "batch_create: bad argument");
    if (opts->saveN < 0 || (opts->saveN > 0 && !opts->zsave)) return fail(LUNA_ERR_BAD_ARG, "batch_create: save points missing");
    const int prec = plans[0]->precision;
    for (int i = 0; i < n; ++i)
        if (!plans[i] || plans[i]->precision != prec) return fail(LUNA_ERR_BAD_ARG, "batch_create: plans must share one precision");
    luna_batch* b = new luna_batch();
    b->n = n;
    b->precision = prec;
    b->plans.assign(plans, plans + n);
    b->opts = *opts;
    b->h.resize(n);
    b->ybuf.resize(n);
    b->ynbuf.resize(n);
    b->steplogs.assign(n, nullptr);
    b->zsave_own.assign(n, nullptr);
    const size_t kel = (prec == LUNA_PREC_FP64) ? sizeof(double2) : sizeof(float2);
    auto bail = [&](int rc) {
        free_all(b->allocs);
        delete b;
        return rc;
    };
    if (opts->saveN > 0) {
        const double* zs = nullptr;
        if (upload(b->allocs, opts->zsave, (size_t)opts->saveN, &zs)) return bail(LUNA_ERR_CUDA);
        b->d_zsave = const_cast<double*>(zs);
    }
    // one slab per instance
    size_t maxsm = 0;
    for (int i = 0; i < n; ++i) {
        LunaInst I = plans[i]->proto;
        const size_t Nw = I.Nw;
        const size_t gsb = (prec == LUNA_PREC_FP64) ? gscr_bytes<double>(I) : gscr_bytes<float>(I);
        size_t off = 0;
        auto carve = [&](size_t bytes) { size_t o = off; off += align_up(bytes, 256); return o; };
        const size_t oy0 = carve(Nw * sizeof(double2));
        const size_t oy = carve(Nw * sizeof(double2)), oyn = carve(Nw * sizeof(double2));
        size_t ok[7];
        for (int j = 0; j < 7; ++j) ok[j] = carve(Nw * kel);
        const size_t oe1 = carve(Nw * sizeof(double2));
        const size_t olz = carve(I.grad ? Nw * sizeof(double2) : 0), ooz = carve(I.grad ? (Nw + 1) * sizeof(double2) : 0);
        // Raman spectrum at ρ(z), rebuilt by the solver in this instance's own buffer
        const size_t ohz = carve((I.grad && I.ramz) ? ((size_t)I.No + 1) * kel : 0);
        const size_t og = carve(gsb);
        const size_t osv = carve((size_t)opts->saveN * Nw * sizeof(double2));
        const size_t olog = carve((size_t)(opts->steplog_cap > 0 ? opts->steplog_cap : 0) * 4 * sizeof(double));
        const size_t ost = carve((size_t)(opts->stats_cap > 0 ? opts->stats_cap : 0) * LUNA_NSTATS * sizeof(double));
        if (opts->stats_cap > 0 && (I.kind != 0 || !I.omega || !I.tgrid || main_len(I) < I.N || I.Nw < 8 || !(I.aeff > 0)))
            return bail(fail(LUNA_ERR_UNSUPPORTED, "batch_create: per-step statistics need a field-resolved grid with "
                                                   "oversampled length >= 2N and the grid's ω, t and Aeff"));
        char* slab = nullptr;
        if (dalloc(b->allocs, &slab, off)) return bail(LUNA_ERR_CUDA);
        I.y0 = (const double2*)(slab + oy0);
        I.y = (double2*)(slab + oy);
        I.yn = (double2*)(slab + oyn);
        for (int j = 0; j < 7; ++j) I.k[j] = slab + ok[j];
        I.e1 = (double2*)(slab + oe1);
        if (I.grad) {
            I.linz = (double2*)(slab + olz);
            I.outz = (double2*)(slab + ooz);
            if (I.ramz) I.resp[I.ramz - 1].H = slab + ohz;
        }
        I.gscr = slab + og;
        I.saves = (double2*)(slab + osv);
        I.zsave = b->d_zsave;
        I.saveN = opts->saveN;
        I.rtol = opts->rtol;
        I.atol = opts->atol;
        I.safety = opts->safety;
        I.max_dt = opts->max_dt;
        I.min_dt = opts->min_dt;
        I.repeat_limit = opts->repeat_limit;
        I.max_steps = opts->max_steps;
        I.steplog = opts->steplog_cap > 0 ? (double*)(slab + olog) : nullptr;
        I.steplog_cap = opts->steplog_cap;
        I.stats = opts->stats_cap > 0 ? (double*)(slab + ost) : nullptr;
        I.stats_cap = opts->stats_cap > 0 ? opts->stats_cap : 0;
        I.nstats = 0;
        I.replay = nullptr;
        I.nreplay = 0;
        if (opts->replay && opts->nreplay > 0) {
            const double* rp = nullptr;
            if (upload(b->allocs, opts->replay, 2 * (size_t)opts->nreplay, &rp)) return bail(LUNA_ERR_CUDA);
            I.replay = rp;
            I.nreplay = opts->nreplay;
        }
        b->steplogs[i] = I.steplog;
        b->ybuf[i] = I.y;
        b->ynbuf[i] = I.yn;
        b->h[i] = I;
        maxsm = std::max(maxsm, (prec == LUNA_PREC_FP64) ? smem_wanted<double>(I) : smem_wanted<float>(I));
    }
    if (dalloc(b->allocs, &b->d_insts, sizeof(LunaInst) * n)) return bail(LUNA_ERR_CUDA);
    if (dalloc(b->allocs, &b->d_counter, sizeof(int))) return bail(LUNA_ERR_CUDA);
    b->smem = (int)std::min<size_t>(maxsm, (size_t)max_smem_optin());
    int dev = 0, nsm = 0, occ = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (prec == LUNA_PREC_FP64) {
        if (cudaFuncSetAttribute(solve_kernel<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, b->smem) != cudaSuccess)
            return bail(fail(LUNA_ERR_CUDA, "batch_create: cannot set shared memory size"));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, solve_kernel<double, double>, LUNA_BLOCK, b->smem);
    } else {
        if (cudaFuncSetAttribute(solve_kernel<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b->smem) != cudaSuccess)
            return bail(fail(LUNA_ERR_CUDA, "batch_create: cannot set shared memory size"));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, solve_kernel<float, float>, LUNA_BLOCK, b->smem);
    }
    if (occ < 1) return bail(fail(LUNA_ERR_CUDA, "batch_create: solver kernel does not fit on an SM"));
    b->grid = std::min(n, nsm * occ);
    if (!(opts->flags & (LUNA_SOLVE_NO_CLUSTERS | LUNA_SOLVE_NO_DIST))) {
        const int rc = (prec == LUNA_PREC_FP64) ? dist_setup<double>(b, opts, nsm) : dist_setup<float>(b, opts, nsm);
        if (rc) return bail(rc);
    }
    if (b->elig.empty() && prec == LUNA_PREC_MIXED && !(opts->flags & LUNA_SOLVE_NO_CLUSTERS)) {
        // Raman clusters for the instances whose Raman buffer alone overflows one CTA
        const int maxs = max_smem_optin();
        std::vector<int> big, reg;
        std::vector<double> cost(n);
        for (int i = 0; i < n; ++i) {
            const LunaInst& I = b->h[i];
            const size_t half = align_up((size_t)(I.No / 2) * sizeof(float2), 256);
            const size_t efac = align_up((size_t)I.Nw * sizeof(float2), 256);
            const bool fits1 = smem_wanted<float>(I) <= (size_t)maxs;
            const bool ok_cl = I.kind == 0 && has_raman(I) && !fits1 && !needs_hilbert(I) && !I.grad &&
                               LUNA_SMALL_BYTES + half + efac <= (size_t)std::min<int>(maxs, b->smem);
            if (ok_cl) big.push_back(i);
            else reg.push_back(i);
            cost[i] = (double)I.No * std::log2((double)I.No) * (has_raman(I) ? 2.0 : 1.0);
        }
        std::stable_sort(reg.begin(), reg.end(), [&](int a, int c) { return cost[a] > cost[c]; });
        if (!big.empty()) {
            if (cudaFuncSetAttribute(solve_kernel_cl<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, b->smem) != cudaSuccess)
                return bail(fail(LUNA_ERR_CUDA, "batch_create: cannot set shared memory size (clusters)"));
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = CL_HELPERS + 1;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.gridDim = dim3((CL_HELPERS + 1) * 32, 1, 1);
            cfg.blockDim = dim3(LUNA_BLOCK, 1, 1);
            cfg.dynamicSmemBytes = b->smem;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int ncl = 0;
            if (cudaOccupancyMaxActiveClusters(&ncl, solve_kernel_cl<float, float>, &cfg) != cudaSuccess || ncl < 1) {
                cudaGetLastError();
                ncl = 0;
            }
            if (ncl >= 1) {
                b->big = big;
                b->reg = reg;
                b->nbig = (int)big.size();
                b->nreg = (int)reg.size();
                // clusters for the big instances (no more than there are), single CTAs
                // on the remaining SMs; both pull the regular instances
                ncl = std::min(ncl, (int)big.size());
                b->cl_grid = (CL_HELPERS + 1) * ncl;
                b->reg_grid = std::max(0, std::min((int)reg.size(), nsm - b->cl_grid));
                std::vector<int> regp(reg);
                if (regp.empty()) regp.push_back(0);  // never read (nreg == 0)
                if (upload(b->allocs, big.data(), big.size(), (const int**)&b->d_big) ||
                    upload(b->allocs, regp.data(), regp.size(), (const int**)&b->d_reg) ||
                    dalloc(b->allocs, &b->d_cl_counters, 3 * sizeof(int)))
                    return bail(LUNA_ERR_CUDA);
            }
        }
    }
    if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream2, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream3, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&b->ev0) != cudaSuccess || cudaEventCreate(&b->ev1) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->evf, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->evj, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->evj3, cudaEventDisableTiming) != cudaSuccess)
        return bail(fail(LUNA_ERR_CUDA, "batch_create: stream/event creation failed"));
    *out = b;
    return LUNA_OK;
}

int luna_b200_batch_upload(luna_batch* b, const double* const* linops, const double* const* y0, const double* z0,
                           const double* dz0, const double* zmax, const double* const* zsave, const double* max_dt) {
    if (!b || !linops || !y0 || !z0 || !dz0 || !zmax) return fail(LUNA_ERR_BAD_ARG, "batch_upload: null argument");
    for (int i = 0; i < b->n; ++i) {
        LunaInst& I = b->h[i];
        const size_t bytes = sizeof(double2) * I.Nw;
        if (zsave && zsave[i] && b->opts.saveN > 0) {
            if (!b->zsave_own[i]) {
                double* zp = nullptr;
                if (dalloc(b->allocs, &zp, sizeof(double) * b->opts.saveN)) return LUNA_ERR_CUDA;
                b->zsave_own[i] = zp;
            }
            CK(cudaMemcpyAsync(b->zsave_own[i], zsave[i], sizeof(double) * b->opts.saveN, cudaMemcpyHostToDevice, b->stream));
            I.zsave = b->zsave_own[i];
        }
        if (max_dt) I.max_dt = max_dt[i];
        // with a pressure gradient L(z) is evaluated on the device and linops[i] is ignored
        if (!I.grad) {
            if (!linops[i]) return fail(LUNA_ERR_BAD_ARG, "batch_upload: null linop for a plan without a pressure gradient");
            if (!I.linop) {
                double2* L = nullptr;
                if (dalloc(b->allocs, &L, bytes)) return LUNA_ERR_CUDA;
                I.linop = L;
            }
            CK(cudaMemcpyAsync((void*)I.linop, linops[i], bytes, cudaMemcpyHostToDevice, b->stream));
        }
        I.y = b->ybuf[i];
        I.yn = b->ynbuf[i];
        CK(cudaMemcpyAsync((void*)I.y0, y0[i], bytes, cudaMemcpyHostToDevice, b->stream));
        I.z0 = z0[i];
        I.dz0 = dz0[i];
        I.zmax = zmax[i];
        I.status = 0;
        I.nsaved = 0;
        I.steps = I.accepted = I.rejected = I.nrhs = 0;
    }
    CK(cudaMemcpyAsync(b->d_insts, b->h.data(), sizeof(LunaInst) * b->n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    return LUNA_OK;
}

int luna_b200_batch_run(luna_batch* b, float* device_ms) {
    if (!b) return fail(LUNA_ERR_BAD_ARG, "batch_run: null batch");
    TwDev tw;
    int rc = get_tw(tw);
    if (rc) return rc;
    // instances restart from y0: restore the per-instance pointers and counters
    CK(cudaMemcpyAsync(b->d_insts, b->h.data(), sizeof(LunaInst) * b->n, cudaMemcpyHostToDevice, b->stream));
    CK(cudaMemsetAsync(b->d_counter, 0, sizeof(int), b->stream));
    if (b->cl_grid > 0) CK(cudaMemsetAsync(b->d_cl_counters, 0, 3 * sizeof(int), b->stream));
    if (b->dist_grid > 0 || b->dist16_grid > 0) CK(cudaMemsetAsync(b->d_cl_counters, 0, 4 * sizeof(int), b->stream));
    CK(cudaEventRecord(b->ev0, b->stream));
    if (b->dist_grid > 0 || b->dist16_grid > 0) {
        rc = (b->precision == LUNA_PREC_FP64) ? dist_launch<double>(b, tw.d) : dist_launch<float>(b, tw.f);
        if (rc) return rc;
    } else if (b->precision == LUNA_PREC_FP64) {
        solve_kernel<double, double><<<b->grid, LUNA_BLOCK, b->smem, b->stream>>>(b->d_insts, b->n, b->d_counter, tw.d, b->smem, nullptr);
    } else if (b->cl_grid > 0) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute at[1];
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = CL_HELPERS + 1;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.gridDim = dim3(b->cl_grid, 1, 1);
        cfg.blockDim = dim3(LUNA_BLOCK, 1, 1);
        cfg.dynamicSmemBytes = b->smem;
        cfg.stream = b->stream;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        int* c = b->d_cl_counters;
        if (b->reg_grid > 0) {
            CK(cudaEventRecord(b->evf, b->stream));
            CK(cudaStreamWaitEvent(b->stream2, b->evf, 0));
        }
        CK(cudaLaunchKernelEx(&cfg, solve_kernel_cl<float, float>, b->d_insts, (const int*)b->d_big, b->nbig, c,
                              (const int*)b->d_reg, b->nreg, c + 1, tw.f, b->smem, c + 2));
        if (b->reg_grid > 0) {
            // the single-CTA solver on the other SMs, submitted after the clusters
            solve_kernel<float, float><<<b->reg_grid, LUNA_BLOCK, b->smem, b->stream2>>>(
                b->d_insts, b->nreg, c + 1, tw.f, b->smem, (const int*)b->d_reg);
            CK(cudaEventRecord(b->evj, b->stream2));
            CK(cudaStreamWaitEvent(b->stream, b->evj, 0));
        }
    } else {
        solve_kernel<float, float><<<b->grid, LUNA_BLOCK, b->smem, b->stream>>>(b->d_insts, b->n, b->d_counter, tw.f, b->smem, nullptr);
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(b->ev1, b->stream));
    CK(cudaEventSynchronize(b->ev1));
    if (device_ms) CK(cudaEventElapsedTime(device_ms, b->ev0, b->ev1));
    return LUNA_OK;
}

int luna_b200_batch_download(luna_batch* b, double* const* saves, double* const* y_out, luna_solve_stats* stats) {
    if (!b) return fail(LUNA_ERR_BAD_ARG, "batch_download: null batch");
    std::vector<LunaInst> res(b->n);
    CK(cudaMemcpyAsync(res.data(), b->d_insts, sizeof(LunaInst) * b->n, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < b->n; ++i) {
        const LunaInst& I = res[i];
        const size_t Nw = I.Nw;
        if (saves && saves[i] && b->opts.saveN > 0)
            CK(cudaMemcpyAsync(saves[i], I.saves, sizeof(double2) * Nw * b->opts.saveN, cudaMemcpyDeviceToHost, b->stream));
        if (y_out && y_out[i]) {
            // the integrator state after the last step: yn when that step was accepted
            CK(cudaMemcpyAsync(y_out[i], I.yn, sizeof(double2) * Nw, cudaMemcpyDeviceToHost, b->stream));
        }
        if (stats) {
            luna_solve_stats& s = stats[i];
            s.status = I.status;
            s.nsaved = I.nsaved;
            s.steps = I.steps;
            s.accepted = I.accepted;
            s.rejected = I.rejected;
            s.nrhs = I.nrhs;
            s.z = I.z;
            s.dz = I.dz;
            s.nstats = I.nstats;
        }
    }
    CK(cudaStreamSynchronize(b->stream));
    return LUNA_OK;
}

int luna_b200_batch_info(luna_batch* b, int* kernels_per_run, int* cluster_instances, int* clusters) {
    if (!b) return fail(LUNA_ERR_BAD_ARG, "batch_info: null batch");
    if (kernels_per_run)
        *kernels_per_run = (b->cl_grid > 0 || b->dist_grid > 0 || b->dist16_grid > 0)
                               ? (b->dist_grid > 0) + (b->dist16_grid > 0) + (b->cl_grid > 0) + (b->reg_grid > 0)
                               : 1;
    if (b->dist_grid > 0 || b->dist16_grid > 0) {
        if (cluster_instances) *cluster_instances = b->ndist + b->ndist16;
        if (clusters) *clusters = b->dist_grid / DIST_R + b->dist16_grid / DIST_R_BIG;
        return LUNA_OK;
    }
    if (cluster_instances) *cluster_instances = (b->cl_grid > 0) ? b->nbig : 0;
    if (clusters) *clusters = b->cl_grid / (CL_HELPERS + 1);
    return LUNA_OK;
}

int luna_b200_batch_set_priority(luna_batch* b, const double* priority) {
    if (!b || !priority) return fail(LUNA_ERR_BAD_ARG, "batch_set_priority: null argument");
    auto by = [&](int a, int c) { return priority[a] > priority[c]; };
    if (!b->elig.empty()) return dist_partition(b, priority);
    if (b->cl_grid == 0) return LUNA_OK;  // single list in index order
    std::stable_sort(b->big.begin(), b->big.end(), by);
    std::stable_sort(b->reg.begin(), b->reg.end(), by);
    CK(cudaMemcpy(b->d_big, b->big.data(), sizeof(int) * b->big.size(), cudaMemcpyHostToDevice));
    if (!b->reg.empty()) CK(cudaMemcpy(b->d_reg, b->reg.data(), sizeof(int) * b->reg.size(), cudaMemcpyHostToDevice));
    return LUNA_OK;
}

int luna_b200_batch_timeline(luna_batch* b, double* begin_end_s, int* sm) {
    if (!b || !begin_end_s) return fail(LUNA_ERR_BAD_ARG, "batch_timeline: null argument");
    std::vector<LunaInst> res(b->n);
    CK(cudaMemcpy(res.data(), b->d_insts, sizeof(LunaInst) * b->n, cudaMemcpyDeviceToHost));
    unsigned long long t0 = ~0ull;
    for (const LunaInst& I : res) t0 = std::min(t0, I.t_begin);
    for (int i = 0; i < b->n; ++i) {
        begin_end_s[2 * i] = (double)(res[i].t_begin - t0) * 1e-9;
        begin_end_s[2 * i + 1] = (double)(res[i].t_end - t0) * 1e-9;
        if (sm) sm[i] = res[i].sm;
    }
    return LUNA_OK;
}

int luna_b200_batch_stats(luna_batch* b, int i, double* stats) {
    if (!b || !stats || i < 0 || i >= b->n) return fail(LUNA_ERR_BAD_ARG, "batch_stats: bad argument");
    if (!b->h[i].stats) return fail(LUNA_ERR_BAD_ARG, "batch_stats: statistics were not requested (stats_cap = 0)");
    CK(cudaMemcpy(stats, b->h[i].stats, sizeof(double) * LUNA_NSTATS * b->h[i].stats_cap, cudaMemcpyDeviceToHost));
    return LUNA_OK;
}

int luna_b200_batch_steplog(luna_batch* b, int i, double* steplog) {
    if (!b || i < 0 || i >= b->n || !steplog || !b->steplogs[i]) return fail(LUNA_ERR_BAD_ARG, "batch_steplog: bad argument");
    CK(cudaMemcpy(steplog, b->steplogs[i], sizeof(double) * 4 * b->opts.steplog_cap, cudaMemcpyDeviceToHost));
    return LUNA_OK;
}

int luna_b200_batch_set_shapes(luna_batch* b, const int* shape) {
    if (!b) return fail(LUNA_ERR_BAD_ARG, "batch_set_shapes: null batch");
    if (!shape) {
        b->shape.clear();
    } else {
        for (int i = 0; i < b->n; ++i)
            if (shape[i] < 0 || shape[i] > 3) return fail(LUNA_ERR_BAD_ARG, "batch_set_shapes: shape must be 0..3");
        b->shape.assign(shape, shape + b->n);
    }
    return LUNA_OK;
}

int luna_b200_batch_set_replay(luna_batch* b, int i, const double* replay, long long nreplay) {
    if (!b || i < 0 || i >= b->n || nreplay < 0 || (nreplay > 0 && !replay))
        return fail(LUNA_ERR_BAD_ARG, "batch_set_replay: bad argument");
    LunaInst& I = b->h[i];
    if (nreplay == 0) {
        I.replay = nullptr;
        I.nreplay = 0;
        return LUNA_OK;
    }
    const double* rp = nullptr;
    if (upload(b->allocs, replay, 2 * (size_t)nreplay, &rp)) return LUNA_ERR_CUDA;
    I.replay = rp;
    I.nreplay = nreplay;
    return LUNA_OK;
}

void luna_b200_batch_destroy(luna_batch* b) {
    if (!b) return;
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->evf) cudaEventDestroy(b->evf);
    if (b->evj) cudaEventDestroy(b->evj);
    if (b->evj3) cudaEventDestroy(b->evj3);
    if (b->stream3) cudaStreamDestroy(b->stream3);
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->stream2) cudaStreamDestroy(b->stream2);
    free_all(b->allocs);
    delete b;
}

int luna_b200_solve(luna_plan* p, const double* linop, double* y_inout, double z0, double dz0, double zmax,
                    const luna_solve_opts* opts, double* saves, double* steplog, luna_solve_stats* stats) {
    if (!p || (!linop && !p->proto.grad) || !y_inout || !opts) return fail(LUNA_ERR_BAD_ARG, "solve: null argument");
    luna_batch* b = nullptr;
    int rc = luna_b200_batch_create(&p, 1, opts, &b);
    if (rc) return rc;
    const double* L[1] = {linop};
    const double* Y[1] = {y_inout};
    rc = luna_b200_batch_upload(b, L, Y, &z0, &dz0, &zmax, nullptr, nullptr);
    if (!rc) rc = luna_b200_batch_run(b, nullptr);
    double* S[1] = {saves};
    double* YO[1] = {y_inout};
    luna_solve_stats st{};
    if (!rc) rc = luna_b200_batch_download(b, S, YO, &st);
    if (!rc && steplog && opts->steplog_cap > 0) rc = luna_b200_batch_steplog(b, 0, steplog);
    luna_b200_batch_destroy(b);
    if (rc) return rc;
    if (stats) *stats = st;
    if (st.status == ST_FIELD_ABOVE_EMAX) return fail(LUNA_FIELD_ABOVE_EMAX, "Field strength exceeds maximum for PPT ionisation rate.");
    if (st.status == ST_REPEAT_LIMIT) return fail(LUNA_REPEAT_LIMIT, "Reached limit for step repetition");
    if (st.status == ST_STEP_BUDGET) return fail(LUNA_STEP_BUDGET, "Step budget exhausted before zmax");
    return LUNA_OK;
}

// ===================================================================== radial transform
}  // extern "C"

// Columns of one tensor-core QDHT tile: 32 gives 2 x ceil(2Nw/128) x Nr/64 CTAs (136 for
// Nw = 1025, Nr = 256 on 148 SMs).
#define RAD_TC_BN 32

struct luna_radial_plan {
    int precision = 0;
    int Nw = 0, Nr = 0;
    luna_plan* col = nullptr;   // grid and responses of one radial column
    LunaInst* d_col = nullptr;  // device copy of the column descriptor
    std::vector<void*> allocs;
    const double* Mi = nullptr;      // [Nr*Nr] row-major QDHT k -> r
    const double* Mf = nullptr;      // [Nr*Nr] row-major QDHT r -> k
    // mixed precision: BF16 hi/lo splits of the QDHT matrices, pre-tiled for the
    // tensor-core products (tc_btile_index<RAD_TC_BN>)
    const __nv_bfloat16 *Mi_t = nullptr, *Mf_t = nullptr;
    const double2* outfac = nullptr; // [Nw*Nr]
    char* gscr = nullptr;            // per-column scratch when a column does not fit in shared memory
    size_t gstride = 0;
    int smem = 0;                    // dynamic shared memory of the column kernels
    void* A = nullptr;               // [Nw*Nr] stage input, then column output
    void* B = nullptr;               // [Nw*Nr] QDHT output
    int* d_flags = nullptr;
    double2* d_Ew = nullptr;
    double2* d_nl = nullptr;
    cudaStream_t stream = nullptr;
    // gas fill gradient (luna_b200_radial_set_gradient): the fill law and tables, and the
    // output factor at the current node
    RadGrad grad{nullptr, nullptr, nullptr};
    double2* ofz = nullptr;
};

namespace {

template <typename Rl>
int rad_column_setup(luna_radial_plan* p) {
    const LunaInst& I = p->col->proto;
    const int maxs = max_smem_optin();
    const size_t want = smem_wanted<Rl>(I);
    p->smem = (int)std::min<size_t>(want, (size_t)maxs);
    if (want > (size_t)maxs) {
        p->gstride = align_up(gscr_bytes<Rl>(I), 256);
        if (dalloc(p->allocs, &p->gscr, p->gstride * p->Nr)) return LUNA_ERR_CUDA;
    }
    // the device maximum, so that plans of different sizes never lower each other's limit
    CK(cudaFuncSetAttribute(rad_column_kernel<Rl>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs));
    CK(cudaFuncSetAttribute(rad_post_kernel<Rl, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs));
    CK(cudaFuncSetAttribute(rad_post_kernel<Rl, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs));
    return LUNA_OK;
}

int rad_grid(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 8); }


uint16_t bf16_rne(float f) {
    uint32_t b;
    memcpy(&b, &f, 4);
    b += 0x7FFFu + ((b >> 16) & 1u);
    return (uint16_t)(b >> 16);
}

float bf16_val(uint16_t h) {
    uint32_t b = (uint32_t)h << 16;
    float f;
    memcpy(&f, &b, 4);
    return f;
}

// Er = A Mi^T or Pk = Pw Mf^T along the radial index of the 2Nw x Nr real view: FP64
// CUDA-core tiles for the plain path, 3xBF16 tensor-core products for the mixed path.
int rad_qdht(luna_radial_plan* p, const void* X, bool fwd, void* Y, const RadState* st, int* flags, cudaStream_t s) {
    const int rows = 2 * p->Nw;
    if (p->precision == LUNA_PREC_FP64) {
        dim3 g((rows + RG_BM - 1) / RG_BM, (p->Nr + RG_BN - 1) / RG_BN);
        rad_gemm_f64<<<g, 256, 0, s>>>((const double*)X, rows, rows, fwd ? p->Mf : p->Mi, (double*)Y, p->Nr, st);
    } else {
        dim3 g((rows + TC_BM - 1) / TC_BM, p->Nr / RAD_TC_BN);
        const int* fin = st ? (const int*)((const char*)st + offsetof(RadState, finished)) : nullptr;
        tc_gemm_3xbf16<RAD_TC_BN><<<g, TC_THREADS, tc_smem_bytes<RAD_TC_BN>(), s>>>(
            (const float*)X, rows, rows, fwd ? p->Mf_t : p->Mi_t, (float*)Y, p->Nr, fin, flags);
    }
    return LUNA_OK;
}

// One transform evaluation: stage input already in A; column output back in A; the
// QDHT r -> k result in B.
template <typename Rl>
int rad_transform(luna_radial_plan* p, const TwTab<Rl>& tw, RadState* st, int* flags, cudaStream_t s) {
    rad_qdht(p, p->A, false, p->B, st, flags, s);
    rad_column_kernel<Rl><<<p->Nr, LUNA_BLOCK, p->smem, s>>>(p->d_col, (const cpx<Rl>*)p->B, (cpx<Rl>*)p->A, tw,
                                                            p->smem, p->gscr, p->gstride, st, flags);
    rad_qdht(p, p->A, true, p->B, st, flags, s);
    return LUNA_OK;
}

template <typename Rl>
int rad_rhs(luna_radial_plan* p, const double2* Ew, double2* nl, cudaStream_t s, double z) {
    TwDev tw;
    int rc = get_tw(tw);
    if (rc) return rc;
    const TwTab<Rl>& t = *reinterpret_cast<const TwTab<Rl>*>(std::is_same<Rl, double>::value ? (const void*)&tw.d : (const void*)&tw.f);
    RadArgs a{p->Nw, p->Nr, nullptr, p->outfac, nullptr, nullptr};
    const size_t n = (size_t)p->Nw * p->Nr;
    if (p->grad.g) {
        // densityfun(z) and normfun(z) of a gas fill gradient
        rad_gradfill_kernel<<<rad_grid(n), 256, 0, s>>>(a, p->grad, -2, z, nullptr, p->ofz);
        a.outfac = p->ofz;
    }
    CK(cudaMemsetAsync(p->d_flags, 0, sizeof(int), s));
    rad_stage_kernel<Rl, double><<<rad_grid(n), 256, 0, s>>>(a, -1, Ew, (cpx<Rl>*)p->A);
    rad_transform<Rl>(p, t, nullptr, p->d_flags, s);
    rad_store_kernel<Rl, double><<<rad_grid(n), 256, 0, s>>>(a, -1, (const cpx<Rl>*)p->B, nl);
    CK(cudaGetLastError());
    return LUNA_OK;
}

}  // namespace

extern "C" {

int luna_b200_radial_plan_create(const luna_grid_desc* g, const luna_resp_desc* resps, int nresp,
                                 const luna_radial_desc* rd, int precision, luna_radial_plan** out) {
    if (!g || !rd || !out || !rd->Mi || !rd->Mf || !rd->outfac)
        return fail(LUNA_ERR_BAD_ARG, "radial_plan_create: null argument");
    if (rd->Nr < 1 || rd->Nr > 4096) return fail(LUNA_ERR_BAD_ARG, "radial_plan_create: Nr must be in 1..4096");
    if (precision != LUNA_PREC_FP64 && precision != LUNA_PREC_MIXED)
        return fail(LUNA_ERR_BAD_ARG, "radial_plan_create: unknown precision");
    if (precision == LUNA_PREC_MIXED && rd->Nr % 64 != 0)
        return fail(LUNA_ERR_UNSUPPORTED, "radial_plan_create: the mixed-precision QDHT needs Nr to be a multiple of 64");
    // the column plan: grid and responses; its output factor is unused (the radial one
    // is applied after the QDHT)
    std::vector<double> ones(2 * (size_t)g->Nw, 0.0);
    for (int k = 0; k < g->Nw; ++k) ones[2 * k] = 1.0;
    luna_grid_desc gc = *g;
    gc.outfac = ones.data();
    luna_plan* col = nullptr;
    int rc = luna_b200_plan_create(&gc, resps, nresp, precision, &col);
    if (rc) return rc;
    luna_radial_plan* p = new luna_radial_plan();
    p->precision = precision;
    p->Nw = g->Nw;
    p->Nr = rd->Nr;
    p->col = col;
    auto bail = [&](int code) {
        free_all(p->allocs);
        luna_b200_plan_destroy(p->col);
        delete p;
        return code;
    };
    const size_t n = (size_t)p->Nw * p->Nr, nn = (size_t)p->Nr * p->Nr;
    const double* tmp = nullptr;
    if (upload(p->allocs, rd->Mi, nn, &p->Mi) || upload(p->allocs, rd->Mf, nn, &p->Mf) ||
        upload(p->allocs, rd->outfac, 2 * n, &tmp))
        return bail(LUNA_ERR_CUDA);
    p->outfac = (const double2*)tmp;
    if (precision == LUNA_PREC_MIXED) {
        // B[n, m] = M[n*Nr + m] (row-major Nr x Nr), split into hi and lo and laid out in
        // the tiles the tensor-core kernel copies whole into shared memory
        std::vector<uint16_t> t(2 * nn);
        const double* src[2] = {rd->Mi, rd->Mf};
        const __nv_bfloat16** dt[2] = {&p->Mi_t, &p->Mf_t};
        const size_t lo_off = (size_t)RAD_TC_BN * TC_KC;
        for (int w = 0; w < 2; ++w) {
            for (int n = 0; n < p->Nr; ++n)
                for (int m = 0; m < p->Nr; ++m) {
                    const double x = src[w][(size_t)n * p->Nr + m];
                    const uint16_t h = bf16_rne((float)x);
                    const size_t i = tc_btile_index<RAD_TC_BN>(n, m, p->Nr);
                    t[i] = h;
                    t[i + lo_off] = bf16_rne((float)(x - (double)bf16_val(h)));
                }
            const uint16_t* d = nullptr;
            if (upload(p->allocs, t.data(), 2 * nn, &d)) return bail(LUNA_ERR_CUDA);
            *dt[w] = (const __nv_bfloat16*)d;
        }
        if (cudaFuncSetAttribute(tc_gemm_3xbf16<RAD_TC_BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 tc_smem_bytes<RAD_TC_BN>()) != cudaSuccess)
            return bail(fail(LUNA_ERR_CUDA, "radial_plan_create: cannot configure the tensor-core kernel"));
    }
    const size_t cb = sizeof(double2);
    if (dalloc(p->allocs, &p->A, cb * n) || dalloc(p->allocs, &p->B, cb * n) || dalloc(p->allocs, &p->d_flags, sizeof(int)) ||
        dalloc(p->allocs, &p->d_col, sizeof(LunaInst)))
        return bail(LUNA_ERR_CUDA);
    if (cudaMemcpy(p->d_col, &col->proto, sizeof(LunaInst), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(LUNA_ERR_CUDA, "radial_plan_create: copy of the column descriptor failed"));
    rc = (precision == LUNA_PREC_FP64) ? rad_column_setup<double>(p) : rad_column_setup<float>(p);
    if (rc) return bail(rc);
    *out = p;
    return LUNA_OK;
}

void luna_b200_radial_plan_destroy(luna_radial_plan* p) {
    if (!p) return;
    if (p->stream) cudaStreamDestroy(p->stream);
    free_all(p->allocs);
    luna_b200_plan_destroy(p->col);
    delete p;
}

int luna_b200_radial_rhs_device(luna_radial_plan* p, double* nl_dev, const double* Ew_dev, double z, void* stream) {
    (void)z;  // constant density and normalisation
    if (!p || !nl_dev || !Ew_dev) return fail(LUNA_ERR_BAD_ARG, "radial_rhs_device: null argument");
    if (p->precision == LUNA_PREC_FP64) return rad_rhs<double>(p, (const double2*)Ew_dev, (double2*)nl_dev, (cudaStream_t)stream, z);
    return rad_rhs<float>(p, (const double2*)Ew_dev, (double2*)nl_dev, (cudaStream_t)stream, z);
}

int luna_b200_radial_set_gradient(luna_radial_plan* p, const luna_gradient_desc* g, const double* kr2,
                                  const double* mu0w) {
    if (!p) return fail(LUNA_ERR_BAD_ARG, "radial_set_gradient: null plan");
    if (!g) {
        p->grad = RadGrad{nullptr, nullptr, nullptr};
        return LUNA_OK;
    }
    const LunaInst& C = p->col->proto;
    for (int i = 0; i < C.nresp; ++i)
        if (C.resp[i].kind == LUNA_RESP_RAMAN && C.resp[i].t2rho)
            return fail(LUNA_ERR_UNSUPPORTED, "radial_set_gradient: a Raman response whose dephasing depends on the "
                                              "density is not available for the radial transform with a gradient");
    if (g->npts < 2 || g->npts > LUNA_GRAD_MAXPTS) return fail(LUNA_ERR_BAD_ARG, "radial_set_gradient: npts out of range");
    if (g->two_point && (g->npts != 2 || g->Z[0] != 0.0))
        return fail(LUNA_ERR_BAD_ARG, "radial_set_gradient: a two-point fill has npts == 2 and starts at z = 0");
    for (int i = 0; i + 1 < g->npts; ++i)
        if (!(g->Z[i + 1] > g->Z[i])) return fail(LUNA_ERR_BAD_ARG, "radial_set_gradient: Z must increase");
    for (int i = 0; i < g->npts; ++i)
        if (!(g->P[i] >= 0) || g->P2[i] != g->P[i] * g->P[i])
            return fail(LUNA_ERR_BAD_ARG, "radial_set_gradient: pressures must be >= 0 with P2 = P*P");
    if (!g->gam || !g->wc || !g->om || !g->ofs || !kr2 || !mu0w || !(g->fd_h12 > 0))
        return fail(LUNA_ERR_BAD_ARG, "radial_set_gradient: null table");
    if (C.kind == 1 && g->env_ref != 0 && g->env_ref != 1)
        return fail(LUNA_ERR_BAD_ARG, "radial_set_gradient: env_ref must be 0 or 1");
    const size_t Nw = (size_t)p->Nw, Nr = (size_t)p->Nr;
    LunaGrad h;
    memset(&h, 0, sizeof(h));
    h.npts = g->npts;
    h.two_point = g->two_point;
    for (int i = 0; i < g->npts; ++i) {
        h.Z[i] = g->Z[i];
        h.P[i] = g->P[i];
        h.P2[i] = g->P2[i];
    }
    h.dens_a = g->dens_a;
    h.dens_b = g->dens_b;
    for (int j = 0; j < 4; ++j) {
        h.fd_xc[j] = g->fd_xc[j];
        h.fd_gam[j] = g->fd_gam[j];
    }
    h.fd_h12 = g->fd_h12;
    h.bref = (C.kind == 1) ? g->env_ref : 0;
    h.ref_xc = g->ref_xc;
    h.ref_gam = g->ref_gam;
    const double* t = nullptr;
    if (upload(p->allocs, g->gam, Nw, &h.gam) || upload(p->allocs, g->wc, Nw, &h.wc) ||
        upload(p->allocs, g->om, Nw, &h.om) || upload(p->allocs, g->ofs, 2 * Nw, &t))
        return LUNA_ERR_CUDA;
    h.ofs = (const double2*)t;
    const LunaGrad* d = nullptr;
    const double *dk = nullptr, *dm = nullptr;
    if (upload(p->allocs, &h, 1, &d) || upload(p->allocs, kr2, Nr, &dk) || upload(p->allocs, mu0w, Nw, &dm))
        return LUNA_ERR_CUDA;
    if (!p->ofz && dalloc(p->allocs, &p->ofz, sizeof(double2) * Nw * Nr)) return LUNA_ERR_CUDA;
    p->grad = RadGrad{d, dk, dm};
    return LUNA_OK;
}

int luna_b200_radial_linop(luna_radial_plan* p, double z, double* linop, double* outfac) {
    if (!p || !linop) return fail(LUNA_ERR_BAD_ARG, "radial_linop: null argument");
    if (!p->grad.g) return fail(LUNA_ERR_BAD_ARG, "radial_linop: the plan has no gas fill gradient");
    const size_t n = (size_t)p->Nw * p->Nr, bytes = sizeof(double2) * n;
    double2* dL = nullptr;
    CK(cudaMalloc(&dL, 2 * bytes));
    RadArgs a{p->Nw, p->Nr, nullptr, nullptr, nullptr, nullptr};
    rad_gradfill_kernel<<<rad_grid(n), 256>>>(a, p->grad, -2, z, dL, dL + n);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpy(linop, dL, bytes, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && outfac) e = cudaMemcpy(outfac, dL + n, bytes, cudaMemcpyDeviceToHost);
    cudaFree(dL);
    if (e != cudaSuccess) return fail(LUNA_ERR_CUDA, std::string("radial_linop: ") + cudaGetErrorString(e));
    return LUNA_OK;
}

int luna_b200_qdht_device(luna_radial_plan* p, void* Y_dev, const void* X_dev, int forward, void* stream) {
    if (!p || !Y_dev || !X_dev || X_dev == Y_dev) return fail(LUNA_ERR_BAD_ARG, "qdht_device: null or aliased argument");
    if (((uintptr_t)X_dev | (uintptr_t)Y_dev) & 7)
        return fail(LUNA_ERR_BAD_ARG, "qdht_device: X and Y must be 8-byte aligned");
    rad_qdht(p, X_dev, forward != 0, Y_dev, nullptr, p->d_flags, (cudaStream_t)stream);
    CK(cudaGetLastError());
    return LUNA_OK;
}

int luna_b200_radial_rhs(luna_radial_plan* p, double* nl, const double* Ew, double z) {
    (void)z;
    if (!p || !nl || !Ew) return fail(LUNA_ERR_BAD_ARG, "radial_rhs: null argument");
    const size_t bytes = sizeof(double2) * p->Nw * p->Nr;
    if (!p->d_Ew) {
        if (dalloc(p->allocs, &p->d_Ew, bytes) || dalloc(p->allocs, &p->d_nl, bytes)) return LUNA_ERR_CUDA;
        CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    }
    CK(cudaMemcpyAsync(p->d_Ew, Ew, bytes, cudaMemcpyHostToDevice, p->stream));
    int rc = (p->precision == LUNA_PREC_FP64) ? rad_rhs<double>(p, p->d_Ew, p->d_nl, p->stream, z)
                                              : rad_rhs<float>(p, p->d_Ew, p->d_nl, p->stream, z);
    if (rc) return rc;
    int fl = 0;
    CK(cudaMemcpyAsync(nl, p->d_nl, bytes, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaMemcpyAsync(&fl, p->d_flags, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    if (fl & (1 << ST_WAIT_TIMEOUT)) return fail(LUNA_WAIT_TIMEOUT, "radial_rhs: a tensor-core wait timed out");
    if (fl & (1 << ST_FIELD_ABOVE_EMAX)) return fail(LUNA_FIELD_ABOVE_EMAX, "Field strength exceeds maximum for PPT ionisation rate.");
    return LUNA_OK;
}

}  // extern "C"

namespace {

// A gas fill gradient of the column transform (radial plans; none for modal plans).
inline RadGrad plan_grad(const luna_radial_plan* p) { return p->grad; }
inline RadGrad plan_grad(const luna_modal_plan*) { return RadGrad{nullptr, nullptr, nullptr}; }

// Device buffers of one column solve (radial or modal transform).
struct RadSolve {
    std::vector<void*> allocs;
    double2 *L = nullptr, *y = nullptr, *yn = nullptr, *e1 = nullptr, *saves = nullptr, *ofz = nullptr;
    void* k[7] = {};
    void** d_k = nullptr;
    double *zsave = nullptr, *steplog = nullptr, *replay = nullptr, *partial = nullptr;
    RadState* st = nullptr;
    LunaInst* opt = nullptr;
    int* h_fin = nullptr;  // pinned
    ~RadSolve() {
        free_all(allocs);
        if (h_fin) cudaFreeHost(h_fin);
    }
};

// RK45.solve_precon with Luna.run's stepfun on an Nw x Nr column state (RK45.jl:19-89,
// Luna.jl:358-391). xform(tw, st, flags, stream) evaluates the transform of the stage
// input in p->A into p->B (before the output factor); `who` names the caller in errors.
template <typename Rl, typename Kt, typename PlanT, typename XF>
int col_solve(PlanT* p, XF&& xform, const char* who, const double* linop, double* y_inout, double z0, double dz0,
              double zmax, const luna_solve_opts* o, double* saves, double* steplog, luna_solve_stats* stats) {
    TwDev tw;
    int rc = get_tw(tw);
    if (rc) return rc;
    const TwTab<Rl>& t = *reinterpret_cast<const TwTab<Rl>*>(std::is_same<Rl, double>::value ? (const void*)&tw.d : (const void*)&tw.f);
    const size_t n = (size_t)p->Nw * p->Nr;
    const size_t cb = sizeof(double2);
    const RadGrad G = plan_grad(p);
    if (!linop && !G.g) return fail(LUNA_ERR_BAD_ARG, std::string(who) + ": null linop");
    RadSolve S;
    if (G.g && dalloc(S.allocs, &S.ofz, cb * n)) return LUNA_ERR_CUDA;
    if (dalloc(S.allocs, &S.L, cb * n) || dalloc(S.allocs, &S.y, cb * n) || dalloc(S.allocs, &S.yn, cb * n) ||
        dalloc(S.allocs, &S.e1, cb * n) || dalloc(S.allocs, &S.st, sizeof(RadState)) ||
        dalloc(S.allocs, &S.opt, sizeof(LunaInst)) || dalloc(S.allocs, &S.d_k, sizeof(void*) * 7))
        return LUNA_ERR_CUDA;
    for (int j = 0; j < 7; ++j)
        if (dalloc(S.allocs, &S.k[j], sizeof(cpx<Kt>) * n)) return LUNA_ERR_CUDA;
    const int nblk = rad_grid(n);
    if (dalloc(S.allocs, &S.partial, sizeof(double) * 3 * nblk)) return LUNA_ERR_CUDA;
    if (o->saveN > 0) {
        if (dalloc(S.allocs, &S.saves, cb * n * o->saveN) || dalloc(S.allocs, &S.zsave, sizeof(double) * o->saveN))
            return LUNA_ERR_CUDA;
        CK(cudaMemcpy(S.zsave, o->zsave, sizeof(double) * o->saveN, cudaMemcpyHostToDevice));
    }
    if (o->steplog_cap > 0 && dalloc(S.allocs, &S.steplog, sizeof(double) * 4 * o->steplog_cap)) return LUNA_ERR_CUDA;
    if (o->replay && o->nreplay > 0) {
        if (dalloc(S.allocs, &S.replay, sizeof(double) * 2 * o->nreplay)) return LUNA_ERR_CUDA;
        CK(cudaMemcpy(S.replay, o->replay, sizeof(double) * 2 * o->nreplay, cudaMemcpyHostToDevice));
    }
    CK(cudaMallocHost(&S.h_fin, sizeof(int)));
    LunaInst I{};
    memset(&I, 0, sizeof(I));
    I.z0 = z0;
    I.dz0 = dz0;
    I.zmax = zmax;
    I.rtol = o->rtol;
    I.atol = o->atol;
    I.safety = o->safety;
    I.max_dt = o->max_dt;
    I.min_dt = o->min_dt;
    I.repeat_limit = o->repeat_limit;
    I.max_steps = o->max_steps;
    I.saveN = o->saveN;
    I.zsave = S.zsave;
    I.saves = S.saves;
    I.steplog = S.steplog;
    I.steplog_cap = S.steplog ? o->steplog_cap : 0;
    I.replay = S.replay;
    I.nreplay = S.replay ? o->nreplay : 0;
    CK(cudaMemcpy(S.opt, &I, sizeof(LunaInst), cudaMemcpyHostToDevice));
    // with a gas fill gradient L(z) is evaluated on the device and linop is ignored
    if (!G.g) CK(cudaMemcpy(S.L, linop, cb * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(S.y, y_inout, cb * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(S.yn, y_inout, cb * n, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(S.d_k, S.k, sizeof(void*) * 7, cudaMemcpyHostToDevice));
    if (!p->stream) CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    cudaStream_t s = p->stream;
    RadArgs a{p->Nw, p->Nr, S.L, G.g ? S.ofz : p->outfac, S.e1, S.st};
    const int eg = rad_grid(n);
    int* flags_dev = (int*)((char*)S.st + offsetof(RadState, flags));
    const int* fin_dev = (const int*)((char*)S.st + offsetof(RadState, finished));
    rad_init_kernel<<<1, 32, 0, s>>>(S.st, S.opt, S.y, S.yn, S.d_k);
    // k1 = f(y0)
    if (G.g) rad_gradfill_kernel<<<eg, 256, 0, s>>>(a, G, -1, 0.0, S.L, S.ofz);
    rad_stage_kernel<Rl, Kt><<<eg, 256, 0, s>>>(a, -1, nullptr, (cpx<Rl>*)p->A);
    xform(t, S.st, flags_dev, s);
    rad_store_kernel<Rl, Kt><<<eg, 256, 0, s>>>(a, -1, (const cpx<Rl>*)p->B, nullptr);
    CK(cudaGetLastError());
    // steps are enqueued in chunks; the loop state on the device says when to stop
    int chunk = 4;
    long long enq = 0;
    const long long cap = (o->max_steps > 0) ? o->max_steps : (long long)1 << 40;
    while (true) {
        for (int q = 0; q < chunk; ++q) {
            rad_begin_kernel<<<1, 32, 0, s>>>(S.st, S.opt);
            for (int sg = 0; sg < 6; ++sg) {
                // L(z) and the output factor at this stage's node (make_prop!, RK45.jl:284-297)
                if (G.g) rad_gradfill_kernel<<<eg, 256, 0, s>>>(a, G, sg, 0.0, S.L, S.ofz);
                rad_stage_kernel<Rl, Kt><<<eg, 256, 0, s>>>(a, sg, nullptr, (cpx<Rl>*)p->A);
                xform(t, S.st, flags_dev, s);
                rad_store_kernel<Rl, Kt><<<eg, 256, 0, s>>>(a, sg, (const cpx<Rl>*)p->B, nullptr);
            }
            rad_combine_kernel<Kt><<<nblk, 256, 0, s>>>(a, S.partial);
            rad_control_kernel<<<1, 256, 0, s>>>(S.st, S.opt, S.partial, nblk);
            rad_post_kernel<Rl, Kt><<<p->Nr, LUNA_BLOCK, p->smem, s>>>(a, p->d_col, S.opt, t, p->smem, p->gscr, p->gstride, G);
        }
        CK(cudaGetLastError());
        enq += chunk;
        CK(cudaMemcpyAsync(S.h_fin, fin_dev, sizeof(int), cudaMemcpyDeviceToHost, s));
        CK(cudaStreamSynchronize(s));
        if (*S.h_fin) break;
        if (enq > cap + 1) return fail(LUNA_ERR_CUDA, std::string(who) + ": loop did not end after max_steps");
        chunk = std::min(chunk * 2, 64);
    }
    // results
    RadState hs;
    LunaInst ho;
    CK(cudaMemcpy(&hs, S.st, sizeof(RadState), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(&ho, S.opt, sizeof(LunaInst), cudaMemcpyDeviceToHost));
    if (saves && o->saveN > 0 && hs.nsaved > 0) CK(cudaMemcpy(saves, S.saves, cb * n * hs.nsaved, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(y_inout, hs.yn, cb * n, cudaMemcpyDeviceToHost));
    if (steplog && S.steplog) CK(cudaMemcpy(steplog, S.steplog, sizeof(double) * 4 * o->steplog_cap, cudaMemcpyDeviceToHost));
    luna_solve_stats r{};
    r.status = hs.c.status;
    r.nsaved = hs.nsaved;
    r.steps = hs.c.steps;
    r.accepted = ho.accepted;
    r.rejected = ho.rejected;
    r.nrhs = 1 + 6 * hs.c.steps;
    r.z = hs.c.tn;
    r.dz = hs.c.dtn;
    if (stats) *stats = r;
    if (r.status == ST_FIELD_ABOVE_EMAX) return fail(LUNA_FIELD_ABOVE_EMAX, "Field strength exceeds maximum for PPT ionisation rate.");
    if (r.status == ST_REPEAT_LIMIT) return fail(LUNA_REPEAT_LIMIT, "Reached limit for step repetition");
    if (r.status == ST_STEP_BUDGET) return fail(LUNA_STEP_BUDGET, "Step budget exhausted before zmax");
    if (r.status == ST_WAIT_TIMEOUT) return fail(LUNA_WAIT_TIMEOUT, std::string(who) + ": a tensor-core wait timed out");
    return LUNA_OK;
}

}  // namespace

extern "C" {

int luna_b200_radial_solve(luna_radial_plan* p, const double* linop, double* y_inout, double z0, double dz0,
                           double zmax, const luna_solve_opts* opts, double* saves, double* steplog,
                           luna_solve_stats* stats) {
    if (!p || (!linop && !p->grad.g) || !y_inout || !opts) return fail(LUNA_ERR_BAD_ARG, "radial_solve: null argument");
    if (opts->saveN < 0 || (opts->saveN > 0 && !opts->zsave)) return fail(LUNA_ERR_BAD_ARG, "radial_solve: save points missing");
    if (p->precision == LUNA_PREC_FP64)
        return col_solve<double, double>(
            p, [p](const TwTab<double>& t, RadState* st, int* fl, cudaStream_t s) { return rad_transform<double>(p, t, st, fl, s); },
            "radial_solve", linop, y_inout, z0, dz0, zmax, opts, saves, steplog, stats);
    return col_solve<float, float>(
        p, [p](const TwTab<float>& t, RadState* st, int* fl, cudaStream_t s) { return rad_transform<float>(p, t, st, fl, s); },
        "radial_solve", linop, y_inout, z0, dz0, zmax, opts, saves, steplog, stats);
}

// ===================================================================== modal transform
}  // extern "C"

struct luna_modal_plan {
    int precision = 0;
    int Nw = 0, Nr = 0;           // Nr: modes (columns of the state)
    int npol = 1, nlevels = 1, nslots = 1, P = 1, nchunk = 1;
    int Mt = 0;  // complex samples of a time buffer: No/2 (real grid) or No (envelope)
    double wlow = 0, rtol = 0, atol = 0, kerr = 0;
    luna_plan* col = nullptr;     // grid and responses of one point
    LunaInst* d_col = nullptr;
    std::vector<void*> allocs;
    const double2* outfac = nullptr;  // [Nr*Nw] crop * ωwin * norm!
    const double* ems = nullptr;      // [nslots*Nr*npol]
    const double* wts = nullptr;      // [nlevels*nslots]
    char* gscr = nullptr;
    size_t gstride = 0;
    int smem = 0;
    void* A = nullptr;   // [Nw*Nr] stage input
    void* B = nullptr;   // [Nw*Nr] integrated transform of the last level
    void* Et = nullptr;  // [Nr*No/2] field samples per mode
    void* G = nullptr;   // [nslots*Nr*No/2] projected polarisation per node
    double* vscr = nullptr;  // two components with plasma: [6*No] doubles per node CTA
    bool vplasma = false;
    ModalState* ms = nullptr;
    int* d_flags = nullptr;
    double2* d_Ew = nullptr;
    double2* d_nl = nullptr;
    cudaStream_t stream = nullptr;
};

namespace {

ModalArgs modal_args(const luna_modal_plan* p, const RadState* st) {
    ModalArgs a;
    a.nmodes = p->Nr;
    a.npol = p->npol;
    a.nslots = p->nslots;
    a.lmax = p->nlevels - 1;
    a.P = p->P;
    a.Mt = p->Mt;
    a.ems = p->ems;
    a.wts = p->wts;
    a.wlow = p->wlow;
    a.rtol = p->rtol;
    a.atol = p->atol;
    a.kerr = p->kerr;
    a.outfac = p->outfac;
    a.Et = p->Et;
    a.G = p->G;
    a.ms = p->ms;
    a.st = st;
    return a;
}

// Transform of the stage input in A into B: fields per mode, then for each cubature level
// its new nodes and its integral; levels after convergence return at once.
template <typename Rl>
int modal_xform(luna_modal_plan* p, const TwTab<Rl>& tw, RadState* st, int* flags, cudaStream_t s) {
    const ModalArgs a = modal_args(p, st);
    modal_time_kernel<Rl><<<p->Nr, LUNA_BLOCK, p->smem, s>>>(p->d_col, (const cpx<Rl>*)p->A, a, tw, p->smem, p->gscr,
                                                             p->gstride);
    for (int l = 0; l < p->nlevels; ++l) {
        const int s0 = (l == 0) ? 0 : (1 << l) - 1;
        const int nn = (l == 0) ? 1 : (1 << l);
        if (p->npol == 1)
            modal_node_kernel<Rl><<<nn, LUNA_BLOCK, p->smem, s>>>(p->d_col, a, s0, tw, p->smem, p->gscr, p->gstride, flags);
        else if (p->vplasma)
            modal_vec_kernel<Rl><<<nn, LUNA_BLOCK, 0, s>>>(p->d_col, a, s0, p->vscr, flags);
        else
            modal_kerr2_kernel<Rl><<<dim3(nn, std::max(1, p->nchunk / nn)), 256, 0, s>>>(p->d_col, a, s0);
        modal_level_kernel<Rl><<<p->Nr, LUNA_BLOCK, p->smem, s>>>(p->d_col, a, l, (cpx<Rl>*)p->B, tw, p->smem, p->gscr,
                                                                  p->gstride);
    }
    return LUNA_OK;
}

template <typename Rl>
int modal_setup(luna_modal_plan* p) {
    const LunaInst& I = p->col->proto;
    const int maxs = max_smem_optin();
    const size_t want = smem_wanted<Rl>(I);
    p->smem = (int)std::min<size_t>(want, (size_t)maxs);
    // time buffer: No/2 sample pairs (real grid) or No complex samples (envelope)
    const int M = (I.kind == 1) ? I.No : I.No / 2;
    p->Mt = M;
    if (want > (size_t)maxs) {
        p->gstride = align_up(gscr_bytes<Rl>(I), 256);
        const int ncta = std::max(p->Nr, 1 << (p->nlevels - 1));
        if (dalloc(p->allocs, &p->gscr, p->gstride * ncta)) return LUNA_ERR_CUDA;
    }
    // split factor of the time buffers: the block transform's when the buffer is in shared
    // memory (the same test as plan_ws), natural order otherwise
    const bool main_smem = LUNA_SMALL_BYTES + align_up((size_t)M * sizeof(cpx<Rl>), 256) <= (size_t)p->smem;
    p->P = main_smem ? fft_nsplit<Rl>(M) : 1;
    p->nchunk = std::max(1, std::min(M / 256, 4 * 148));
    if (dalloc(p->allocs, &p->Et, sizeof(cpx<Rl>) * (size_t)p->Nr * M) ||
        dalloc(p->allocs, &p->G, sizeof(cpx<Rl>) * (size_t)p->nslots * p->Nr * M))
        return LUNA_ERR_CUDA;
    // the largest level has 2^(nlevels - 1) new nodes, one CTA each
    if (p->vplasma && dalloc(p->allocs, &p->vscr, sizeof(double) * 6 * (size_t)I.No * ((size_t)1 << (p->nlevels - 1))))
        return LUNA_ERR_CUDA;
    CK(cudaFuncSetAttribute(modal_time_kernel<Rl>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs));
    CK(cudaFuncSetAttribute(modal_node_kernel<Rl>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs));
    CK(cudaFuncSetAttribute(modal_level_kernel<Rl>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs));
    CK(cudaFuncSetAttribute(rad_post_kernel<Rl, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs));
    CK(cudaFuncSetAttribute(rad_post_kernel<Rl, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, maxs));
    return LUNA_OK;
}

template <typename Rl>
int modal_rhs(luna_modal_plan* p, const double2* Ew, double2* nl, cudaStream_t s) {
    TwDev tw;
    int rc = get_tw(tw);
    if (rc) return rc;
    const TwTab<Rl>& t = *reinterpret_cast<const TwTab<Rl>*>(std::is_same<Rl, double>::value ? (const void*)&tw.d : (const void*)&tw.f);
    RadArgs a{p->Nw, p->Nr, nullptr, p->outfac, nullptr, nullptr};
    const size_t n = (size_t)p->Nw * p->Nr;
    CK(cudaMemsetAsync(p->d_flags, 0, sizeof(int), s));
    rad_stage_kernel<Rl, double><<<rad_grid(n), 256, 0, s>>>(a, -1, Ew, (cpx<Rl>*)p->A);
    modal_xform<Rl>(p, t, nullptr, p->d_flags, s);
    rad_store_kernel<Rl, double><<<rad_grid(n), 256, 0, s>>>(a, -1, (const cpx<Rl>*)p->B, nl);
    CK(cudaGetLastError());
    return LUNA_OK;
}

}  // namespace

extern "C" {

int luna_b200_modal_plan_create(const luna_grid_desc* g, const luna_resp_desc* resps, int nresp,
                                const luna_modal_desc* md, int precision, luna_modal_plan** out) {
    if (!g || !md || !out || !md->ems || !md->wts || !md->outfac || (nresp > 0 && !resps))
        return fail(LUNA_ERR_BAD_ARG, "modal_plan_create: null argument");
    if (md->nmodes < 1 || md->nmodes > LUNA_MODAL_MAX_MODES)
        return fail(LUNA_ERR_BAD_ARG, "modal_plan_create: nmodes must be in 1..LUNA_MODAL_MAX_MODES");
    if (md->npol != 1 && md->npol != 2) return fail(LUNA_ERR_BAD_ARG, "modal_plan_create: npol must be 1 or 2");
    if (md->nlevels < 1 || md->nlevels > LUNA_MODAL_MAX_LEVELS)
        return fail(LUNA_ERR_BAD_ARG, "modal_plan_create: nlevels must be in 1..LUNA_MODAL_MAX_LEVELS");
    if (!(md->rtol >= 0) || !(md->atol >= 0)) return fail(LUNA_ERR_BAD_ARG, "modal_plan_create: negative tolerance");
    if (precision != LUNA_PREC_FP64 && precision != LUNA_PREC_MIXED)
        return fail(LUNA_ERR_BAD_ARG, "modal_plan_create: unknown precision");
    double kerr = 0;
    bool vplasma = false;
    for (int i = 0; i < nresp; ++i) {
        const int k = resps[i].kind;
        // RamanPolar on a modal field: the scalar case only (Nonlinear.jl:284-293, "vector
        // Raman not yet implemented"); the analytic-signal forms are not available here
        if (k == LUNA_RESP_RAMAN_NOTHG || k == LUNA_RESP_KERR_FIELD_NOTHG)
            return fail(LUNA_ERR_UNSUPPORTED, "modal_plan_create: the no-THG response forms are not available for the modal transform");
        if (md->npol == 2 && k == LUNA_RESP_RAMAN)
            return fail(LUNA_ERR_UNSUPPORTED, "modal_plan_create: vector Raman is not implemented (as in the reference)");
        if (md->npol == 2 && k != LUNA_RESP_KERR_FIELD && k != LUNA_RESP_KERR_ENV && k != LUNA_RESP_PLASMA_PPT &&
            k != LUNA_RESP_PLASMA_ADK)
            return fail(LUNA_ERR_UNSUPPORTED, "modal_plan_create: two polarisation components support Kerr and plasma");
        // (Kerr_env_thg is a scalar form: two components take Kerr_env, KerrVectorEnv!)
        if (g->kind == 1 && (k == LUNA_RESP_PLASMA_PPT || k == LUNA_RESP_PLASMA_ADK))
            return fail(LUNA_ERR_UNSUPPORTED, "modal_plan_create: no plasma response for envelope fields (as in the reference)");
        if (md->npol == 2 && (k == LUNA_RESP_PLASMA_PPT || k == LUNA_RESP_PLASMA_ADK)) {
            if (vplasma) return fail(LUNA_ERR_UNSUPPORTED, "modal_plan_create: at most one plasma response");
            vplasma = true;
        }
        if (k == LUNA_RESP_KERR_FIELD || k == LUNA_RESP_KERR_ENV) kerr += resps[i].coef;
    }
    // the point plan: grid and responses; its output factor is unused (the modal one is
    // applied after the cubature)
    std::vector<double> ones(2 * (size_t)g->Nw, 0.0);
    for (int k = 0; k < g->Nw; ++k) ones[2 * k] = 1.0;
    luna_grid_desc gc = *g;
    gc.outfac = ones.data();
    luna_plan* col = nullptr;
    int rc = luna_b200_plan_create(&gc, resps, nresp, precision, &col);
    if (rc) return rc;
    luna_modal_plan* p = new luna_modal_plan();
    p->precision = precision;
    p->Nw = g->Nw;
    p->Nr = md->nmodes;
    p->npol = md->npol;
    p->nlevels = md->nlevels;
    p->nslots = (2 << (md->nlevels - 1)) - 1;
    p->wlow = md->wlow;
    p->rtol = md->rtol;
    p->atol = md->atol;
    p->kerr = kerr;
    p->vplasma = vplasma;
    p->col = col;
    auto bail = [&](int code) {
        free_all(p->allocs);
        luna_b200_plan_destroy(p->col);
        delete p;
        return code;
    };
    const size_t n = (size_t)p->Nw * p->Nr;
    const double* tmp = nullptr;
    if (upload(p->allocs, md->outfac, 2 * n, &tmp) ||
        upload(p->allocs, md->ems, (size_t)p->nslots * p->Nr * p->npol, &p->ems) ||
        upload(p->allocs, md->wts, (size_t)p->nlevels * p->nslots, &p->wts))
        return bail(LUNA_ERR_CUDA);
    p->outfac = (const double2*)tmp;
    const size_t cb = sizeof(double2);
    if (dalloc(p->allocs, &p->A, cb * n) || dalloc(p->allocs, &p->B, cb * n) || dalloc(p->allocs, &p->d_flags, sizeof(int)) ||
        dalloc(p->allocs, &p->ms, sizeof(ModalState)) || dalloc(p->allocs, &p->d_col, sizeof(LunaInst)))
        return bail(LUNA_ERR_CUDA);
    if (cudaMemset(p->ms, 0, sizeof(ModalState)) != cudaSuccess ||
        cudaMemcpy(p->d_col, &col->proto, sizeof(LunaInst), cudaMemcpyHostToDevice) != cudaSuccess)
        return bail(fail(LUNA_ERR_CUDA, "modal_plan_create: initialising the device state failed"));
    rc = (precision == LUNA_PREC_FP64) ? modal_setup<double>(p) : modal_setup<float>(p);
    if (rc) return bail(rc);
    *out = p;
    return LUNA_OK;
}

void luna_b200_modal_plan_destroy(luna_modal_plan* p) {
    if (!p) return;
    if (p->stream) cudaStreamDestroy(p->stream);
    free_all(p->allocs);
    luna_b200_plan_destroy(p->col);
    delete p;
}

int luna_b200_modal_rhs_device(luna_modal_plan* p, double* nl_dev, const double* Ew_dev, double z, void* stream) {
    (void)z;  // constant density
    if (!p || !nl_dev || !Ew_dev) return fail(LUNA_ERR_BAD_ARG, "modal_rhs_device: null argument");
    if (p->precision == LUNA_PREC_FP64) return modal_rhs<double>(p, (const double2*)Ew_dev, (double2*)nl_dev, (cudaStream_t)stream);
    return modal_rhs<float>(p, (const double2*)Ew_dev, (double2*)nl_dev, (cudaStream_t)stream);
}

int luna_b200_modal_rhs(luna_modal_plan* p, double* nl, const double* Ew, double z, int* nevals) {
    (void)z;
    if (!p || !nl || !Ew) return fail(LUNA_ERR_BAD_ARG, "modal_rhs: null argument");
    const size_t bytes = sizeof(double2) * p->Nw * p->Nr;
    if (!p->d_Ew) {
        if (dalloc(p->allocs, &p->d_Ew, bytes) || dalloc(p->allocs, &p->d_nl, bytes)) return LUNA_ERR_CUDA;
        CK(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking));
    }
    CK(cudaMemcpyAsync(p->d_Ew, Ew, bytes, cudaMemcpyHostToDevice, p->stream));
    int rc = (p->precision == LUNA_PREC_FP64) ? modal_rhs<double>(p, p->d_Ew, p->d_nl, p->stream)
                                              : modal_rhs<float>(p, p->d_Ew, p->d_nl, p->stream);
    if (rc) return rc;
    int fl = 0, nev = 0;
    CK(cudaMemcpyAsync(nl, p->d_nl, bytes, cudaMemcpyDeviceToHost, p->stream));
    CK(cudaMemcpyAsync(&fl, p->d_flags, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    CK(cudaMemcpyAsync(&nev, &p->ms->nevals, sizeof(int), cudaMemcpyDeviceToHost, p->stream));
    CK(cudaStreamSynchronize(p->stream));
    if (nevals) *nevals = nev;
    if (fl & (1 << ST_FIELD_ABOVE_EMAX)) return fail(LUNA_FIELD_ABOVE_EMAX, "Field strength exceeds maximum for PPT ionisation rate.");
    return LUNA_OK;
}

int luna_b200_modal_solve(luna_modal_plan* p, const double* linop, double* y_inout, double z0, double dz0, double zmax,
                          const luna_solve_opts* opts, double* saves, double* steplog, luna_solve_stats* stats) {
    if (!p || !linop || !y_inout || !opts) return fail(LUNA_ERR_BAD_ARG, "modal_solve: null argument");
    if (opts->saveN < 0 || (opts->saveN > 0 && !opts->zsave)) return fail(LUNA_ERR_BAD_ARG, "modal_solve: save points missing");
    if (p->precision == LUNA_PREC_FP64)
        return col_solve<double, double>(
            p, [p](const TwTab<double>& t, RadState* st, int* fl, cudaStream_t s) { return modal_xform<double>(p, t, st, fl, s); },
            "modal_solve", linop, y_inout, z0, dz0, zmax, opts, saves, steplog, stats);
    return col_solve<float, float>(
        p, [p](const TwTab<float>& t, RadState* st, int* fl, cudaStream_t s) { return modal_xform<float>(p, t, st, fl, s); },
        "modal_solve", linop, y_inout, z0, dz0, zmax, opts, saves, steplog, stats);
}

// ---------------------------------------------------------------- allocation-free RHS
// The scratch lives in static device memory. Host code must not pass the symbol itself to
// a kernel (on the host it names a host-side shadow); its device address is resolved with
// cudaGetSymbolAddress once per device and cached.
static __device__ __align__(256) unsigned char g_noalloc_scratch[LUNA_NOALLOC_SCRATCH_BYTES];

}  // extern "C"

namespace {
std::mutex g_na_mu;
std::map<int, void*> g_na_ptr;

int noalloc_scratch(void** out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_na_mu);
    auto it = g_na_ptr.find(dev);
    if (it != g_na_ptr.end()) {
        *out = it->second;
        return LUNA_OK;
    }
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
        return fail(LUNA_ERR_CUDA, std::string("noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
    g_na_ptr[dev] = p;
    *out = p;
    return LUNA_OK;
}

// twiddle tables of the current device without creating them (plan creation did)
int find_tw(TwDev& out) {
    int dev = 0;
    CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_tw_mu);
    auto it = g_tw.find(dev);
    if (it == g_tw.end()) return fail(LUNA_ERR_BAD_ARG, "noalloc: no plan was created on this device");
    out = it->second;
    return LUNA_OK;
}
}  // namespace

// The kernel's status word is documented as the public codes
static_assert(ST_OK == LUNA_OK && ST_FIELD_ABOVE_EMAX == LUNA_FIELD_ABOVE_EMAX,
              "rhs_kernel_noalloc writes ST_* values where the header promises LUNA_* codes");

// The instance description travels as a kernel parameter, so the call needs no device copy.
template <typename Rl>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
rhs_kernel_noalloc(const LunaInst I, const double2* Ew, double2* nl, TwTab<Rl> tw, int smem_bytes, int* status) {
    extern __shared__ __align__(256) char smem[];
    Ws<Rl> w;
    plan_ws<Rl>(I, smem, smem_bytes, w, tw);
    if (threadIdx.x == 0) *w.flag = 0;
    __syncthreads();
    const cpx<double>* E = reinterpret_cast<const cpx<double>*>(Ew);
    cpx<double>* o = reinterpret_cast<cpx<double>*>(nl);
    rhs<Rl>(I, w, [&](int k) { return E[k]; }, [&](int k, cpx<double> v) { o[k] = v; });
    __syncthreads();
    if (threadIdx.x == 0 && status) *status = (*w.flag & (1 << ST_FIELD_ABOVE_EMAX)) ? ST_FIELD_ABOVE_EMAX : ST_OK;
}

extern "C" int luna_b200_rhs_device_noalloc(luna_plan* p, double* nl_dev, const double* Ew_dev, double z,
                                            void* stream, int* status_dev) {
    (void)z;  // constant density and effective area: the transform does not depend on z
    if (!p || !nl_dev || !Ew_dev) return fail(LUNA_ERR_BAD_ARG, "rhs_device_noalloc: null argument");
    if (p->proto.grad)
        return fail(LUNA_ERR_UNSUPPORTED, "rhs_device_noalloc: plans with a pressure gradient need a per-plan "
                                          "buffer for the z-dependent normalisation; use luna_b200_rhs_device");
    LunaInst I = p->proto;
    const size_t need = (p->precision == LUNA_PREC_FP64) ? gscr_bytes<double>(I) : gscr_bytes<float>(I);
    if (need > (size_t)LUNA_NOALLOC_SCRATCH_BYTES)
        return fail(LUNA_ERR_UNSUPPORTED, "rhs_device_noalloc: the plan needs " + std::to_string(need) +
                                              " bytes of scratch, more than LUNA_NOALLOC_SCRATCH_BYTES (" +
                                              std::to_string((size_t)LUNA_NOALLOC_SCRATCH_BYTES) + ")");
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    TwDev tw;
    rc = find_tw(tw);
    if (rc) return rc;
    I.gscr = scratch;
    const int maxs = max_smem_optin();
    cudaStream_t st = (cudaStream_t)stream;
    if (p->precision == LUNA_PREC_FP64) {
        int sm = (int)std::min<size_t>(smem_wanted<double>(I), (size_t)maxs);
        CK(cudaFuncSetAttribute(rhs_kernel_noalloc<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        rhs_kernel_noalloc<double><<<1, LUNA_BLOCK, sm, st>>>(I, (const double2*)Ew_dev, (double2*)nl_dev, tw.d, sm, status_dev);
    } else {
        int sm = (int)std::min<size_t>(smem_wanted<float>(I), (size_t)maxs);
        CK(cudaFuncSetAttribute(rhs_kernel_noalloc<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm));
        rhs_kernel_noalloc<float><<<1, LUNA_BLOCK, sm, st>>>(I, (const double2*)Ew_dev, (double2*)nl_dev, tw.f, sm, status_dev);
    }
    CK(cudaGetLastError());
    return LUNA_OK;
}
