// Radially symmetric free-space transform (TransRadial, NonlinearRHS.jl:466-474) and its
// RK45 loop on the device.
//
// The reference evaluates, per right-hand side,
//   irfft along t -> QDHT k->r along the radial index -> responses per radial column
//   -> time window -> QDHT r->k -> rfft along t -> crop -> ωwin(-iω)/(2 normfun).
// The QDHT is a real Nr x Nr matrix acting on the radial index and the FFT acts on the
// time/frequency index, so the two commute. Here both matrix products act on the
// frequency side, on the Nw x Nr complex arrays (2*Nw real rows instead of No):
//   A  = exp(L d) (y + dt sum B k)               stage kernel   (elementwise, Nw x Nr)
//   Er = A Mi^T                                  QDHT k->r      (GEMM, 2Nw x Nr x Nr)
//   Pw = crop(rfft(towin * P(irfft(pad Er))))    column kernel  (one CTA per radial column)
//   Pk = Pw Mf^T                                 QDHT r->k      (GEMM)
//   k_{s+1} = Pk outfac / exp(L d)               store kernel   (elementwise)
// Arrays are column-major Nw x Nr complex, the layout of Julia's Matrix{ComplexF64}:
// element (ω, c) at c*Nw + ω.
//
// The integrator state (RK45.jl:128-226 with Luna.run's stepfun) lives in a RadState in
// global memory; each step is a fixed launch sequence whose kernels return at once after
// the loop has finished, so the host can enqueue several steps before it looks.
#pragma once
#include "uppe.cuh"

namespace luna {

struct RadState {
    Ctl c;               // t, tn, dt, dtn, err, errlast, ok, done, status, repeated, steps; k[7]
    double2* y;          // state at t
    double2* yn;         // proposal at tn (after acceptance: the next state)
    double dprop;        // tn - t at the start of the step: k1 <- exp(L dprop) k1
    int finished;        // the loop has ended: every kernel returns immediately
    int swap_y;          // y <- yn at the next step start
    int nsaved;          // save points taken so far
    int save_lo, save_hi;  // save points taken by the current accepted step
    int flags;           // status bits raised by the column kernels
};

struct RadArgs {
    int Nw, Nr;
    const double2* L;       // [Nw*Nr] linear operator (of the current node with a gas fill gradient)
    const double2* outfac;  // [Nw*Nr] crop * ωwin * (-iω) / (2 normfun) (x ρ(z) with a gradient)
    double2* e1;            // [Nw*Nr] exp(L dt) of the last stage with node 1
    RadState* st;
};

// ------------------------------------------------------------------ gas fill gradient
// make_linop(grid, q, nfun) for radial symmetry (LinearOps.jl:174-226) and norm_radial
// (NonlinearRHS.jl:494-524) with nfun(ω; z) = sqrt(1 + γ(ω) ρ(z)), ρ(z) the density law of a
// luna_gradient_desc (Capillary.gradient, Capillary.jl:306-337):
//   k2(ω) = (n ω/c)^2 on sidx (0 elsewhere), βsq = k2 - k_r^2,
//   L = -i (sqrt(βsq) - β1(z) ω), or -i (-β1 ω) - min(sqrt|βsq|, 200) when βsq < 0,
//   + i β(ω0; z) on an envelope grid without THG, β1(z) the 4-point central difference of
//   x/c n(x; z) at ω0 (h = 1e-4 ω0); normfun = sqrt(βsq)/(μ0 ω) for ω != 0 and βsq > 0, else 1;
// each in IEEE-rounded operations in the order of the host restatement. The responses'
// coefficients are given for ρ = 1; ρ(z) scales the output factor.
struct RadGrad {
    const LunaGrad* g;  // fill law, γ and ω/c on sidx (wc = 0 elsewhere), ω (om), ofs, fd tables
    const double* kr2;  // [Nr] k_r^2 of the QDHT
    const double* mw;   // [Nw] μ0 ω
};

// (ρ(z), β1(z), β(ω0; z)) into out[3]
__device__ __forceinline__ void rad_grad_scalars(const LunaGrad* g, double z, double* out) {
    const double rho = grad_density(g, z);
    double f[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) f[j] = __dmul_rn(g->fd_xc[j], __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(g->fd_gam[j], rho))));
    const double num = __dadd_rn(__dsub_rn(__dadd_rn(-f[0], __dmul_rn(8.0, f[1])), __dmul_rn(8.0, f[2])), f[3]);
    out[0] = rho;
    out[1] = __ddiv_rn(num, g->fd_h12);
    out[2] = g->bref ? __dmul_rn(g->ref_xc, __dsqrt_rn(__dadd_rn(1.0, __dmul_rn(g->ref_gam, rho)))) : 0.0;
}

// L and the output factor of element (ω index i, k index c)
__device__ __forceinline__ void rad_grad_elem(const RadGrad& G, int i, int c, const double* sc, cpx<double>& L,
                                              cpx<double>& of) {
    const LunaGrad* g = G.g;
    const double rho = sc[0], b1 = sc[1];
    const double wc = __ldg(g->wc + i), w = __ldg(g->om + i);
    double k2 = 0.0;
    if (wc != 0.0) {
        const double nk = __dmul_rn(__dsqrt_rn(__dadd_rn(1.0, __dmul_rn(__ldg(g->gam + i), rho))), wc);
        k2 = __dmul_rn(nk, nk);
    }
    const double bsq = __dsub_rn(k2, __ldg(G.kr2 + c));
    const double bw = __dmul_rn(b1, w);
    double re, im;
    if (bsq < 0) {
        re = -fmin(__dsqrt_rn(-bsq), 200.0);
        im = bw;
    } else {
        re = 0.0;
        im = -__dsub_rn(__dsqrt_rn(bsq), bw);
    }
    if (g->bref) im = __dadd_rn(im, sc[2]);
    L = mk<double>(re, im);
    const double2 o = __ldg(g->ofs + i);
    double ox = __dmul_rn(rho, o.x), oy = __dmul_rn(rho, o.y);
    if (w != 0.0 && bsq > 0) {
        const double nr = __ddiv_rn(__dsqrt_rn(bsq), __ldg(G.mw + i));
        ox = __ddiv_rn(ox, nr);
        oy = __ddiv_rn(oy, nr);
    }
    of = mk<double>(ox, oy);
}

// L(z) and the output factor at z over the whole Nw x Nr array, z the node of stage s of
// the current step (s >= 0), the current z of the loop (s == -1) or zfix (s == -2).
__global__ void __launch_bounds__(256) rad_gradfill_kernel(RadArgs a, RadGrad G, int s, double zfix, double2* Lz,
                                                           double2* ofz) {
    const RadState* st = a.st;
    if (s != -2 && st->finished) return;
    __shared__ double sc[3];
    if (threadIdx.x == 0) {
        double z = zfix;
        if (s >= 0) z = __dadd_rn(st->c.t, __dmul_rn(c_nodes[s], st->c.dt));
        else if (s == -1) z = st->c.t;
        rad_grad_scalars(G.g, z, sc);
    }
    __syncthreads();
    const size_t n = (size_t)a.Nw * a.Nr;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
        const int c = (int)(e / a.Nw), i = (int)(e - (size_t)c * a.Nw);
        cpx<double> L, of;
        rad_grad_elem(G, i, c, sc, L, of);
        if (Lz) reinterpret_cast<cpx<double>*>(Lz)[e] = L;
        reinterpret_cast<cpx<double>*>(ofz)[e] = of;
    }
}

// ------------------------------------------------------------------ elementwise stages
// Stage input A = exp(L d) (y + dt sum_j B[s][j] k_j) (the load of the fused mode-averaged
// kernel, one element per thread); s < 0: A = src (a plain right-hand side evaluation).
template <typename Rl, typename Kt>
__global__ void __launch_bounds__(256) rad_stage_kernel(RadArgs a, int s, const double2* src, cpx<Rl>* A) {
    const RadState* st = a.st;
    if (st && st->finished) return;
    const size_t n = (size_t)a.Nw * a.Nr;
    const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, di = (size_t)gridDim.x * blockDim.x;
    if (s < 0) {
        const cpx<double>* y = reinterpret_cast<const cpx<double>*>(src ? src : (const double2*)st->y);
        for (size_t i = i0; i < n; i += di) A[i] = cvt<Rl>(y[i]);
        return;
    }
    const double t0 = st->c.t, dt = st->c.dt;
    const double d = __dsub_rn(__dadd_rn(t0, __dmul_rn(c_nodes[s], dt)), t0);  // node - t, as rounded
    const bool propk1 = (s == 0) && (st->dprop != 0.0);
    const cpx<double>* y = reinterpret_cast<const cpx<double>*>(st->y);
    const cpx<double>* L = reinterpret_cast<const cpx<double>*>(a.L);
    cpx<double>* e1 = reinterpret_cast<cpx<double>*>(a.e1);
    void* k[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) k[j] = st->c.k[j];
    const double c0 = dt * c_B[s][0];
    for (size_t i = i0; i < n; i += di) {
        const cpx<Rl> f = expLd<Rl>(L[i], d);
        if (s == 4) e1[i] = cvt<double>(f);
        cpx<double> k1 = KT<Kt>::ld(k[0], i);
        if (propk1) {
            k1 = k1 * e1[i];
            KT<Kt>::st(k[0], i, k1);
        }
        cpx<double> acc = y[i];
        acc = acc + scale(c0, k1);
        for (int j = 1; j <= s; ++j) {
            const double bj = c_B[s][j];
            if (bj != 0) acc = acc + scale(dt * bj, KT<Kt>::ld(k[j], i));
        }
        A[i] = cvt<Rl>(cvt<double>(f) * acc);
    }
}

// k_{s+1} = Pk * outfac / exp(L d); s < 0: dst = Pk * outfac (k1 of the first step, or the
// output of a plain right-hand side evaluation).
template <typename Rl, typename Kt>
__global__ void __launch_bounds__(256) rad_store_kernel(RadArgs a, int s, const cpx<Rl>* Pk, void* dst) {
    const RadState* st = a.st;
    if (st && st->finished) return;
    const size_t n = (size_t)a.Nw * a.Nr;
    const size_t i0 = (size_t)blockIdx.x * blockDim.x + threadIdx.x, di = (size_t)gridDim.x * blockDim.x;
    const cpx<double>* of = reinterpret_cast<const cpx<double>*>(a.outfac);
    if (s < 0) {
        void* o = dst ? dst : st->c.k[0];
        for (size_t i = i0; i < n; i += di) KT<Kt>::st(o, i, cvt<double>(Pk[i]) * of[i]);
        return;
    }
    const double t0 = st->c.t, dt = st->c.dt;
    const double d = __dsub_rn(__dadd_rn(t0, __dmul_rn(c_nodes[s], dt)), t0);
    const cpx<double>* L = reinterpret_cast<const cpx<double>*>(a.L);
    void* kout = st->c.k[s + 1];
    for (size_t i = i0; i < n; i += di) {
        const cpx<Rl> f = expLd<Rl>(L[i], d);
        KT<Kt>::st(kout, i, (cvt<double>(Pk[i]) * of[i]) * inv_fac<Rl>(f));
    }
}

// ------------------------------------------------------------------ QDHT products (FP64)
// C[r, n] = sum_m A[r + m*lda] * B[n*K + m] for r < rows, n < N (= K = Nr): the QDHT
// matrix B (row-major Nr x Nr) applied along the radial index of the column-major
// 2Nw x Nr real view of a complex Nw x Nr array. 64 x 64 output tile per CTA, 16-deep
// K slices staged in shared memory, 4 x 4 outputs per thread.
#define RG_BM 64
#define RG_BN 64
#define RG_BK 16
__global__ void __launch_bounds__(256) rad_gemm_f64(const double* __restrict__ A, int lda, int rows,
                                                    const double* __restrict__ B, double* __restrict__ C, int K,
                                                    const RadState* st) {
    if (st && st->finished) return;
    __shared__ double As[2][RG_BK][RG_BM];
    __shared__ double Bs[2][RG_BK][RG_BN + 1];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int r0 = blockIdx.x * RG_BM, n0 = blockIdx.y * RG_BN;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
    // loaders: A slice 16 x 64 (4 per thread, coalesced along r); B slice 64 x 16 (4 per
    // thread, coalesced along m)
    auto load = [&](int kb, int buf) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = tid + 256 * q;
            const int kk = e >> 6, rr = e & 63;
            const int r = r0 + rr, m = kb + kk;
            As[buf][kk][rr] = (r < rows && m < K) ? A[(size_t)m * lda + r] : 0.0;
            const int nn = e >> 4, mk = e & 15;
            const int nB = n0 + nn, mB = kb + mk;
            Bs[buf][mk][nn] = (nB < K && mB < K) ? B[(size_t)nB * K + mB] : 0.0;
        }
    };
    load(0, 0);
    __syncthreads();
    int buf = 0;
    for (int kb = 0; kb < K; kb += RG_BK) {
        if (kb + RG_BK < K) load(kb + RG_BK, buf ^ 1);
#pragma unroll
        for (int kk = 0; kk < RG_BK; ++kk) {
            double av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) av[i] = As[buf][kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) bv[j] = Bs[buf][kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = r0 + tx + 16 * i;
        if (r >= rows) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int n = n0 + ty + 16 * j;
            if (n < K) C[(size_t)n * lda + r] = acc[i][j];
        }
    }
}

// ------------------------------------------------------------------ per-column responses
// One CTA per radial column n: Pw[:, n] = crop-free rfft(towin * P(irfft(pad Er[:, n])))
// (to_time!, Et_to_Pt!, towin, to_freq! of TransRadial on one column, which the reference
// applies column by column, NonlinearRHS.jl:137-141; the pad scale and 1/No are in
// I.in_scale, the crop scale in the output factor). The column is the mode-averaged
// transform of a plan whose output factor is one: field-resolved grids with every response
// form (Raman and the analytic-signal forms included) and envelope grids (fft/ifft with
// copy_scale_both! padding). The FP32 form is compiled for two CTAs per SM (64 registers,
// a few hundred bytes of spills), so that 256 columns run in one wave on 148 SMs instead
// of two (4.5 % less time per right-hand side at Nr = 256, No = 4096).
template <typename Rl>
__global__ void __launch_bounds__(LUNA_BLOCK, sizeof(Rl) == 4 ? 2 : 1)
rad_column_kernel(const LunaInst* inst, const cpx<Rl>* Er, cpx<Rl>* Pw, TwTab<Rl> tw, int smem_bytes,
                  char* gscr, size_t gstride, RadState* st, int* flags) {
    extern __shared__ __align__(256) char smem[];
    if (st && st->finished) return;
    const LunaInst& I = *inst;
    const int c = blockIdx.x;
    Ws<Rl> w;
    plan_ws<Rl>(I, smem, smem_bytes, w, tw, gscr ? gscr + (size_t)c * gstride : nullptr);
    if (threadIdx.x == 0) *w.flag = 0;
    __syncthreads();
    const cpx<Rl>* E = Er + (size_t)c * I.Nw;
    cpx<Rl>* o = Pw + (size_t)c * I.Nw;
    rhs<Rl>(I, w, [&](int k) { return cvt<double>(E[k]); }, [&](int k, cpx<double> X) { o[k] = cvt<Rl>(X); });
    if (threadIdx.x == 0 && *w.flag) atomicOr(flags, *w.flag);
}

// ------------------------------------------------------------------ step bookkeeping
__global__ void rad_init_kernel(RadState* st, LunaInst* opt, double2* y, double2* yn, void* const* k) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Ctl& c = st->c;
    for (int j = 0; j < 7; ++j) c.k[j] = k[j];
    c.t = c.tn = opt->z0;
    c.dt = c.dtn = opt->dz0;
    c.err = c.errlast = 0;
    c.ok = 0;
    c.done = 0;
    c.status = 0;
    c.repeated = 0;
    c.steps = 0;
    st->y = y;
    st->yn = yn;
    st->dprop = 0;
    st->finished = 0;
    st->swap_y = 0;
    st->nsaved = 0;
    st->save_lo = st->save_hi = 0;
    st->flags = 0;
    opt->accepted = opt->rejected = 0;
}

// Loop head of RK45.solve / evaluate! (RK45.jl:43-78, 209-223).
__global__ void rad_begin_kernel(RadState* st, const LunaInst* opt) {
    if (threadIdx.x != 0 || blockIdx.x != 0 || st->finished) return;
    Ctl& c = st->c;
    if (!(c.tn <= opt->zmax) || c.done) {
        st->finished = 1;
        return;
    }
    if (st->swap_y) {
        double2* t = st->y;
        st->y = st->yn;
        st->yn = t;
    }
    st->dprop = c.tn - c.t;
    c.dt = c.dtn;
    c.t = c.tn;
}

// yn = y + dt sum b5_j k_j and the three sums of the weak norm, per block (fixed
// partition, so the reduction order does not change from run to run).
template <typename Kt>
__global__ void __launch_bounds__(256) rad_combine_kernel(RadArgs a, double* partial) {
    const RadState* st = a.st;
    if (st->finished) return;
    __shared__ double red[3 * 8];
    const size_t n = (size_t)a.Nw * a.Nr;
    const double dt = st->c.dt;
    const cpx<double>* y = reinterpret_cast<const cpx<double>*>(st->y);
    cpx<double>* yn = reinterpret_cast<cpx<double>*>(st->yn);
    void* k[7];
    double cb5[7], cer[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) {
        k[j] = st->c.k[j];
        cb5[j] = dt * c_b5[j];
        cer[j] = c_b5[j] - c_b4[j];
    }
    double sy = 0, syn = 0, se = 0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
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
    sy = warp_sum(sy);
    syn = warp_sum(syn);
    se = warp_sum(se);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) {
        red[wid] = sy;
        red[8 + wid] = syn;
        red[16 + wid] = se;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a0 = 0, a1 = 0, a2 = 0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            a0 += red[i];
            a1 += red[8 + i];
            a2 += red[16 + i];
        }
        partial[3 * blockIdx.x + 0] = a0;
        partial[3 * blockIdx.x + 1] = a1;
        partial[3 * blockIdx.x + 2] = a2;
    }
}

// Weak norm, PI controller and bookkeeping (the same code as the fused solver), FSAL
// rotation and the save points the accepted step covers. One CTA of 256 threads: thread t
// sums the partials t, t+256, ... in order, then a fixed-order tree (deterministic).
__global__ void __launch_bounds__(256) rad_control_kernel(RadState* st, LunaInst* opt, const double* partial,
                                                          int nblocks) {
    if (st->finished) return;
    __shared__ double red[3][256];
    double sy = 0, syn = 0, se = 0;
    for (int b = threadIdx.x; b < nblocks; b += 256) {
        sy += partial[3 * b];
        syn += partial[3 * b + 1];
        se += partial[3 * b + 2];
    }
    red[0][threadIdx.x] = sy;
    red[1][threadIdx.x] = syn;
    red[2][threadIdx.x] = se;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    sy = red[0][0];
    syn = red[1][0];
    se = red[2][0];
    Ctl& c = st->c;
    control_step(*opt, c, sy, syn, se, st->flags);
    if (st->flags & (1 << ST_WAIT_TIMEOUT)) {
        c.status = ST_WAIT_TIMEOUT;
        c.done = 1;
    }
    if (c.done && c.status != 0) {
        st->finished = 1;
        return;
    }
    if (c.ok) {
        void* t = c.k[0];  // FSAL: ks[1] <- ks[7]
        c.k[0] = c.k[6];
        c.k[6] = t;
        int hi = st->nsaved;
        while (hi < opt->saveN && opt->zsave[hi] <= c.tn) ++hi;
        st->save_lo = st->nsaved;
        st->save_hi = hi;
        st->nsaved = hi;
        st->swap_y = 1;
    } else {
        st->save_lo = st->save_hi = st->nsaved;
        st->swap_y = 0;
    }
}

// After the controller, per k column: accepted -> prop!_maybe + stepfun window filter on
// yn and the dense-output saves (Luna.jl:366-372, RK45.jl:249-268, Output.jl:490-502);
// rejected -> yn = y.
template <typename Rl, typename Kt>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
rad_post_kernel(RadArgs a, const LunaInst* inst, const LunaInst* opt, TwTab<Rl> tw, int smem_bytes, char* gscr,
                size_t gstride, RadGrad G) {
    extern __shared__ __align__(256) char smem[];
    const RadState* st = a.st;
    if (st->finished) return;
    const LunaInst& I = *inst;
    const int c = blockIdx.x, Nw = a.Nw;
    const size_t off = (size_t)c * Nw;
    double2* y = st->y + off;
    double2* yn = st->yn + off;
    if (!st->c.ok) {
        for (int i = threadIdx.x; i < Nw; i += LUNA_BLOCK) yn[i] = y[i];
        return;
    }
    Ws<Rl> w;
    plan_ws<Rl>(I, smem, smem_bytes, w, tw, gscr ? gscr + (size_t)c * gstride : nullptr);
    stepfun_filter<Rl>(I, w, yn, a.e1 + off);
    void* kc[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) kc[j] = (char*)st->c.k[j] + off * sizeof(cpx<Kt>);
    for (int si = st->save_lo; si < st->save_hi; ++si) {
        if (G.g) {
            // L of this column at the save point (a gas fill gradient: prop! to z_i with
            // linop!(z_i), RK45.jl:284-297); the node buffer is free until the next step
            __shared__ double sc[3];
            __syncthreads();
            if (threadIdx.x == 0) rad_grad_scalars(G.g, opt->zsave[si], sc);
            __syncthreads();
            cpx<double>* Lc = reinterpret_cast<cpx<double>*>(const_cast<double2*>(a.L)) + off;
            for (int i = threadIdx.x; i < Nw; i += LUNA_BLOCK) {
                cpx<double> L, of;
                rad_grad_elem(G, i, c, sc, L, of);
                Lc[i] = L;
            }
            __syncthreads();
        }
        interpolate_row<Rl, Kt>(Nw, a.L + off, st->c, opt->zsave[si], kc, y, yn,
                                opt->saves + (size_t)si * Nw * a.Nr + off);
    }
}

}  // namespace luna
