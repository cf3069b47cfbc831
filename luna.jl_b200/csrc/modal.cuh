// Modal transform (TransModal with full=false, NonlinearRHS.jl:148-302) on the device.
//
// The reference evaluates, per transverse point r of a p-adaptive Clenshaw-Curtis rule on
// (0, a) (Cubature.pcubature_v, NonlinearRHS.jl:294-298):
//   Erω = Emω Ems(r) -> irfft -> responses -> towin -> rfft -> crop -> ωwin -> norm!
//   -> Prω Ems(r)^T, times 2πr,
// and sums the points with the rule's weights, doubling the rule until the L2 difference
// from the previous rule meets the tolerance. Everything between the two mode products is
// linear except the responses, and the mode products act on the mode index only, so the
// sum over points moves to the time samples:
//   E_m(t)  = irfft(pad Emω[:, m])                          time kernel, one CTA per mode
//   g_s,m(t) = sum_p Ems[s][m][p] towin P_p(sum_m' Ems[s][m'][p] E_m'(t))
//                                                           node kernel, per new node s
//   X_l,m   = rfft(sum_s W[l][s] g_s,m)                     level kernel, one CTA per mode
// with W[l][s] the level-l weight of node s (2πr and the half-width included). Each level
// costs one forward transform per mode instead of two transforms per point. The level
// kernel compares X_l (times the output factor crop ωwin norm!) with the previous level,
// and the last of its CTAs decides whether the cubature has converged; the kernels of the
// remaining levels then return at once. X of the last level taken is left in B for the
// store kernel of the column solver (radial.cuh), which applies the output factor.
//
// Time samples are kept in the buffer order of the block transforms (slot i of a buffer
// holds the sample pair n with Swz(split_pos(n)) == i), the same in every kernel, so node
// and level sums are plain element-wise loops over the buffers.
#pragma once
#include "radial.cuh"

namespace luna {

#define MODAL_MAX_MODES 16
#define MODAL_MAX_LEVELS 9

struct ModalState {
    int done;         // the cubature of the current right-hand side has ended
    int nevals;       // integrand evaluations it took (2^(l+1) + 1 at level l)
    unsigned ticket;  // level-kernel CTAs that have finished the current level
    int pad;
    double err;       // L2 error estimate of the last level
    double part[2 * MODAL_MAX_MODES];  // per mode: sum |F_l - F_{l-1}|^2, sum |F_l|^2
};

struct ModalArgs {
    int nmodes, npol, nslots, lmax, P;
    int Mt;                 // complex samples of a time buffer: No/2 pairs (real grid), No (envelope)
    const double* ems;      // [nslots][nmodes][npol] normalised mode fields at the nodes
    const double* wts;      // [lmax + 1][nslots] node weights of each level's rule
    double wlow;            // weight of node 0 in the midpoint rule (level 0's comparison)
    double rtol, atol;      // pcubature reltol / abstol on the L2 norm
    double kerr;            // sum of the Kerr coefficients (vector Kerr)
    const double2* outfac;  // [nmodes * Nw] crop * ωwin * norm!
    void* Et;               // [nmodes][M] field samples per mode (buffer order)
    void* G;                // [nslots][nmodes][M] projected polarisation per node
    ModalState* ms;
    const RadState* st;     // loop state of a solve (null for a plain evaluation)
};

__device__ __forceinline__ bool modal_skip(const ModalArgs& a) {
    return (a.st && a.st->finished) || a.ms->done;
}

// E_m(t) for every mode: to_time! of column m of the stage input A.
template <typename Rl>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
modal_time_kernel(const LunaInst* inst, const cpx<Rl>* A, ModalArgs a, TwTab<Rl> tw, int smem_bytes,
                  char* gscr, size_t gstride) {
    extern __shared__ __align__(256) char smem[];
    if (a.st && a.st->finished) return;
    const LunaInst& I = *inst;
    const int c = blockIdx.x;
    if (c == 0 && threadIdx.x == 0) {
        a.ms->done = 0;
        a.ms->ticket = 0;
    }
    Ws<Rl> w;
    plan_ws<Rl>(I, smem, smem_bytes, w, tw, gscr ? gscr + (size_t)c * gstride : nullptr);
    const int M = I.No / 2, Mt = a.Mt;
    const cpx<Rl>* E = A + (size_t)c * I.Nw;
    int P;
    auto ld = [&](int k) { return cvt<double>(E[k]); };
    // envelope grids: to_time! with copy_scale_both! (NonlinearRHS.jl:16-32), No complex samples
    cpx<Rl>* x = (I.kind == 1) ? env_to_time<Rl>(I, w, ld, &P) : c2r_to_time<Rl>(w, M, I.Nw, ld, &P);
    cpx<Rl>* out = reinterpret_cast<cpx<Rl>*>(a.Et) + (size_t)c * Mt;
    for (int i = threadIdx.x; i < Mt; i += LUNA_BLOCK) out[i] = x[i];
}

// One polarisation component: one CTA per new node. The point's field is built in the
// CTA's transform buffer and the responses of the mode-averaged kernel (Kerr, plasma) and
// the time window are applied in place; the result times each mode's field at the node
// goes to G.
template <typename Rl>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
modal_node_kernel(const LunaInst* inst, ModalArgs a, int slot0, TwTab<Rl> tw, int smem_bytes, char* gscr,
                  size_t gstride, int* flags) {
    extern __shared__ __align__(256) char smem[];
    if (modal_skip(a)) return;
    const LunaInst& I = *inst;
    const int slot = slot0 + blockIdx.x;
    Ws<Rl> w;
    plan_ws<Rl>(I, smem, smem_bytes, w, tw, gscr ? gscr + (size_t)blockIdx.x * gstride : nullptr);
    if (threadIdx.x == 0) *w.flag = 0;
    const int M = a.Mt, nm = a.nmodes;
    const int P = buf_split<Rl>(w.main_alt, M);
    const double* e = a.ems + (size_t)slot * nm;
    const cpx<Rl>* Et = reinterpret_cast<const cpx<Rl>*>(a.Et);
    cpx<Rl>* x = w.main;
    for (int i = threadIdx.x; i < M; i += LUNA_BLOCK) {
        double sx = 0, sy = 0;
        for (int m = 0; m < nm; ++m) {
            const cpx<Rl> v = Et[(size_t)m * M + i];
            sx += e[m] * (double)v.x;
            sy += e[m] * (double)v.y;
        }
        x[i] = mk<Rl>((Rl)sx, (Rl)sy);
    }
    __syncthreads();
    if (I.kind == 1) pointwise_env<Rl>(I, w, x, P, I.in_scale);  // Kerr_env(_thg), RamanPolarEnv
    else pointwise_real<Rl>(I, w, x, M, P, I.in_scale);
    cpx<Rl>* G = reinterpret_cast<cpx<Rl>*>(a.G) + (size_t)slot * nm * M;
    for (int m = 0; m < nm; ++m) {
        const double em = e[m];
        for (int i = threadIdx.x; i < M; i += LUNA_BLOCK) {
            const cpx<Rl> v = x[i];
            G[(size_t)m * M + i] = mk<Rl>((Rl)(em * (double)v.x), (Rl)(em * (double)v.y));
        }
    }
    __syncthreads();
    if (threadIdx.x == 0 && *w.flag && flags) atomicOr(flags, *w.flag);
}

// Two polarisation components, Kerr only (KerrVector!, Nonlinear.jl:12-21): element-wise,
// so each new node is spread over gridDim.y CTAs.
template <typename Rl>
__global__ void __launch_bounds__(256) modal_kerr2_kernel(const LunaInst* inst, ModalArgs a, int slot0) {
    if (modal_skip(a)) return;
    const LunaInst& I = *inst;
    const int slot = slot0 + blockIdx.x;
    const int M = a.Mt, nm = a.nmodes, P = a.P, Lb = M / P;
    const double* e = a.ems + (size_t)slot * nm * 2;
    const cpx<Rl>* Et = reinterpret_cast<const cpx<Rl>*>(a.Et);
    cpx<Rl>* G = reinterpret_cast<cpx<Rl>*>(a.G) + (size_t)slot * nm * M;
    const double sc = I.in_scale, kc = a.kerr;
    if (I.kind == 1) {
        // KerrVectorEnv! (Nonlinear.jl:52-63): slot i holds the complex sample n
        for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < M; i += gridDim.y * blockDim.x) {
            const int sp = Swz<Rl>::f(i);
            const int n = (sp % Lb) * P + sp / Lb;
            cpx<double> ex = mk<double>(0, 0), ey = mk<double>(0, 0);
            for (int m = 0; m < nm; ++m) {
                const cpx<double> v = cvt<double>(Et[(size_t)m * M + i]);
                ex = ex + scale(e[2 * m], v);
                ey = ey + scale(e[2 * m + 1], v);
            }
            ex = scale(sc, ex);
            ey = scale(sc, ey);
            const double ax = abs2(ex), ay = abs2(ey), f = 0.75 * kc, tw = __ldg(I.towin + n);
            const cpx<double> px = scale(f, scale(ax + 2.0 / 3 * ay, ex) + scale(1.0 / 3, conj(ex) * (ey * ey)));
            const cpx<double> py = scale(f, scale(ay + 2.0 / 3 * ax, ey) + scale(1.0 / 3, conj(ey) * (ex * ex)));
            for (int m = 0; m < nm; ++m)
                G[(size_t)m * M + i] = cvt<Rl>(scale(tw, scale(e[2 * m], px) + scale(e[2 * m + 1], py)));
        }
        return;
    }
    for (int i = blockIdx.y * blockDim.x + threadIdx.x; i < M; i += gridDim.y * blockDim.x) {
        const int sp = Swz<Rl>::f(i);            // the swizzle is its own inverse
        const int n = (sp % Lb) * P + sp / Lb;   // inverse of split_pos
        double ex0 = 0, ey0 = 0, ex1 = 0, ey1 = 0;
        for (int m = 0; m < nm; ++m) {
            const cpx<Rl> v = Et[(size_t)m * M + i];
            const double fx = e[2 * m], fy = e[2 * m + 1];
            ex0 += fx * (double)v.x;
            ey0 += fy * (double)v.x;
            ex1 += fx * (double)v.y;
            ey1 += fy * (double)v.y;
        }
        ex0 *= sc;
        ey0 *= sc;
        ex1 *= sc;
        ey1 *= sc;
        const double tw0 = __ldg(I.towin + 2 * n), tw1 = __ldg(I.towin + 2 * n + 1);
        const double f0 = kc * (ex0 * ex0 + ey0 * ey0), f1 = kc * (ex1 * ex1 + ey1 * ey1);
        const double px0 = f0 * ex0 * tw0, py0 = f0 * ey0 * tw0;
        const double px1 = f1 * ex1 * tw1, py1 = f1 * ey1 * tw1;
        for (int m = 0; m < nm; ++m) {
            const double fx = e[2 * m], fy = e[2 * m + 1];
            G[(size_t)m * M + i] = mk<Rl>((Rl)(fx * px0 + fy * py0), (Rl)(fx * px1 + fy * py1));
        }
    }
}

// Exclusive prefix of v over the CTA's threads (thread order) and the total; sh holds
// LUNA_WARPS doubles.
__device__ __forceinline__ double cta_exscan(double v, double* sh, double& total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) sh[wid] = x;
    __syncthreads();
    if (wid == 0) {
        double t = (lane < LUNA_WARPS) ? sh[lane] : 0.0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < LUNA_WARPS) sh[lane] = t;
    }
    __syncthreads();
    const double base = wid ? sh[wid - 1] : 0.0;
    total = sh[LUNA_WARPS - 1];
    __syncthreads();
    return base + x - v;
}

// Maths.cumtrapz! (Maths.jl:323-328) of v[0..n) on one CTA, written as the prefix sum
// out[j] = dt (S_j - (v_0 + v_j)/2), S_j = v_0 + ... + v_j, each thread a contiguous run.
__device__ __forceinline__ void cta_cumtrapz(const double* v, double* out, int n, double dt, double* sh) {
    const int C = (n + LUNA_BLOCK - 1) / LUNA_BLOCK;
    const int b = threadIdx.x * C, e = min(n, b + C);
    const double v0 = v[0];  // read before the scan's barriers: out may alias v
    double s = 0;
    for (int j = b; j < e; ++j) s += v[j];
    double tot;
    double pre = cta_exscan(s, sh, tot);
    for (int j = b; j < e; ++j) {
        pre += v[j];
        out[j] = dt * (pre - 0.5 * (v0 + v[j]));
    }
    __syncthreads();
}

// Two polarisation components with the plasma response (PlasmaVector!, Nonlinear.jl:144-162)
// and vector Kerr (KerrVector!, Nonlinear.jl:12-21): one CTA per new node. The node's field
// (Ex, Ey) in natural time order, the rate of |E| = hypot(Ex, Ey) and the ionisation fraction,
// the phase integrands and currents of both components, their cumulative integrals, then
// the polarisation times the time window projected on each mode's field at the node.
// Scratch: 6 No doubles per CTA in global memory (vs).
template <typename Rl>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
modal_vec_kernel(const LunaInst* inst, ModalArgs a, int slot0, double* vscr, int* flags) {
    __shared__ double sh[LUNA_WARPS];
    __shared__ int flag;
    if (modal_skip(a)) return;
    const LunaInst& I = *inst;
    const int slot = slot0 + blockIdx.x;
    const int M = I.No / 2, No = I.No, nm = a.nmodes, P = a.P, Lb = M / P;
    const int tid = threadIdx.x;
    if (tid == 0) flag = 0;
    int ip = -1;
    for (int i = 0; i < I.nresp; ++i)
        if (I.resp[i].kind == LUNA_RESP_PLASMA_PPT || I.resp[i].kind == LUNA_RESP_PLASMA_ADK) ip = i;
    const LunaResp& r = I.resp[ip];
    const double* e = a.ems + (size_t)slot * nm * 2;
    const cpx<Rl>* Et = reinterpret_cast<const cpx<Rl>*>(a.Et);
    cpx<Rl>* G = reinterpret_cast<cpx<Rl>*>(a.G) + (size_t)slot * nm * M;
    double* ex = vscr + (size_t)blockIdx.x * 6 * No;
    double* ey = ex + No;
    double* rt = ey + No;   // rate, then Px
    double* fr = rt + No;   // cumulative rate, the fraction, then Py
    double* jx = fr + No;   // phase integrand and current, x
    double* jy = jx + No;   // phase integrand and current, y
    const double sc = I.in_scale, kc = a.kerr, dt = r.dt;
    __syncthreads();
    // the node's field in natural order (buffer slot i holds the sample pair n)
    for (int i = tid; i < M; i += LUNA_BLOCK) {
        const int sp = Swz<Rl>::f(i);
        const int n = (sp % Lb) * P + sp / Lb;
        double x0 = 0, y0 = 0, x1 = 0, y1 = 0;
        for (int m = 0; m < nm; ++m) {
            const cpx<Rl> v = Et[(size_t)m * M + i];
            const double fx = e[2 * m], fy = e[2 * m + 1];
            x0 += fx * (double)v.x;
            y0 += fy * (double)v.x;
            x1 += fx * (double)v.y;
            y1 += fy * (double)v.y;
        }
        ex[2 * n] = x0 * sc;
        ey[2 * n] = y0 * sc;
        ex[2 * n + 1] = x1 * sc;
        ey[2 * n + 1] = y1 * sc;
    }
    __syncthreads();
    for (int j = tid; j < No; j += LUNA_BLOCK) {
        const double Em = hypot(ex[j], ey[j]);
        rt[j] = (r.kind == LUNA_RESP_PLASMA_PPT) ? ppt_rate<double>(r, Em, &flag) : adk_rate<double>(r, Em);
    }
    __syncthreads();
    cta_cumtrapz(rt, fr, No, dt, sh);
    for (int j = tid; j < No; j += LUNA_BLOCK) {
        const double f = r.preion + 1.0 - exp(-fr[j]);
        fr[j] = f;
        jx[j] = f * r.eratio * ex[j];
        jy[j] = f * r.eratio * ey[j];
    }
    __syncthreads();
    // J = cumtrapz(phase) + ionpot rate (1 - fraction)/|E|^2 E per component, in place
    cta_cumtrapz(jx, jx, No, dt, sh);
    cta_cumtrapz(jy, jy, No, dt, sh);
    for (int j = tid; j < No; j += LUNA_BLOCK) {
        const double Em = hypot(ex[j], ey[j]);
        const double f = fr[j];
        if (fabs(Em) > 0) {
            const double pre = r.ionpot * rt[j] * (1.0 - f) / (Em * Em);
            jx[j] += pre * ex[j];
            jy[j] += pre * ey[j];
        }
    }
    __syncthreads();
    cta_cumtrapz(jx, rt, No, dt, sh);  // Px (the rates are no longer needed)
    cta_cumtrapz(jy, fr, No, dt, sh);  // Py
    const double coef = r.coef;
    for (int i = tid; i < M; i += LUNA_BLOCK) {
        const int sp = Swz<Rl>::f(i);
        const int n = (sp % Lb) * P + sp / Lb;
        double pxy[2][2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = 2 * n + h;
            const double Ex = ex[j], Ey = ey[j];
            const double fk = kc * (Ex * Ex + Ey * Ey);
            const double tw = __ldg(I.towin + j);
            pxy[h][0] = (fk * Ex + coef * rt[j]) * tw;
            pxy[h][1] = (fk * Ey + coef * fr[j]) * tw;
        }
        for (int m = 0; m < nm; ++m) {
            const double fx = e[2 * m], fy = e[2 * m + 1];
            G[(size_t)m * M + i] = mk<Rl>((Rl)(fx * pxy[0][0] + fy * pxy[0][1]), (Rl)(fx * pxy[1][0] + fy * pxy[1][1]));
        }
    }
    __syncthreads();
    if (tid == 0 && flag && flags) atomicOr(flags, flag);
}

// Level l of the rule for mode c: X_l = rfft(sum_s W[l][s] g_s,c) into B (level 0 first
// puts the midpoint rule there), the two L2 sums against the previous level, and the
// convergence decision by the last CTA to finish (Cubature's L2 error norm).
template <typename Rl>
__global__ void __launch_bounds__(LUNA_BLOCK, 1)
modal_level_kernel(const LunaInst* inst, ModalArgs a, int l, cpx<Rl>* B, TwTab<Rl> tw, int smem_bytes,
                   char* gscr, size_t gstride) {
    extern __shared__ __align__(256) char smem[];
    if (modal_skip(a)) return;
    const LunaInst& I = *inst;
    const int c = blockIdx.x;
    Ws<Rl> w;
    plan_ws<Rl>(I, smem, smem_bytes, w, tw, gscr ? gscr + (size_t)c * gstride : nullptr);
    const int M = a.Mt, Nw = I.Nw, nm = a.nmodes;
    const int ns = (2 << l) - 1;  // interior nodes of level l
    const double* wl = a.wts + (size_t)l * a.nslots;
    const cpx<Rl>* G = reinterpret_cast<const cpx<Rl>*>(a.G);
    cpx<Rl>* Bc = B + (size_t)c * Nw;
    const cpx<double>* of = reinterpret_cast<const cpx<double>*>(a.outfac) + (size_t)c * Nw;
    double se = 0, sv = 0;
    for (int pass = (l == 0) ? 0 : 1; pass < 2; ++pass) {
        cpx<Rl>* x = w.main;
        for (int i = threadIdx.x; i < M; i += LUNA_BLOCK) {
            double sx = 0, sy = 0;
            if (pass == 0) {
                const cpx<Rl> v = G[(size_t)c * M + i];
                sx = a.wlow * (double)v.x;
                sy = a.wlow * (double)v.y;
            } else {
                for (int s = 0; s < ns; ++s) {
                    const double ws = wl[s];
                    const cpx<Rl> v = G[((size_t)s * nm + c) * M + i];
                    sx += ws * (double)v.x;
                    sy += ws * (double)v.y;
                }
            }
            x[i] = mk<Rl>((Rl)sx, (Rl)sy);
        }
        __syncthreads();
        const bool cmp = pass == 1;
        auto st = [&](int k, cpx<double> X) {
            if (cmp) {
                const cpx<double> o = ldg(of + k);
                se += abs2((X - cvt<double>(Bc[k])) * o);
                sv += abs2(X * o);
            }
            Bc[k] = cvt<Rl>(X);
        };
        if (I.kind == 1) env_to_freq<Rl>(I, w, x, st);
        else r2c_to_freq<Rl>(w, x, M, Nw, st);
    }
    double unused = 0;
    block_sum3(se, sv, unused, w.red);
    if (threadIdx.x == 0) {
        ModalState* ms = a.ms;
        ms->part[2 * c] = se;
        ms->part[2 * c + 1] = sv;
        __threadfence();
        const unsigned tk = atomicAdd(&ms->ticket, 1u);
        if (tk == (unsigned)nm - 1) {
            __threadfence();
            const volatile double* pp = ms->part;
            double e2 = 0, v2 = 0;
            for (int m = 0; m < nm; ++m) {
                e2 += pp[2 * m];
                v2 += pp[2 * m + 1];
            }
            const double err = sqrt(e2), val = sqrt(v2);
            ms->err = err;
            ms->nevals = (2 << l) + 1;
            if (err <= a.atol || err <= a.rtol * val || l >= a.lmax) ms->done = 1;
            ms->ticket = 0;
        }
    }
}

}  // namespace luna
