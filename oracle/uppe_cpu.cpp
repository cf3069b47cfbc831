// FP64 C++ restatement of the mode-averaged UPPE hot path (test infrastructure and the timed
// CPU baseline; never part of the product path).
//
// It follows the numpy restatement in uppe.py operation for operation, which in turn follows
// Luna.jl v0.6.2: to_time!/to_freq! (NonlinearRHS.jl:16-53), TransModeAvg (NonlinearRHS.jl:
// 362-373), Et_to_Pt! (NonlinearRHS.jl:121-126), Kerr_field (Nonlinear.jl:8-34),
// PlasmaCumtrapz with the PPT spline or ADK rate (Nonlinear.jl:88-177, Ionisation.jl:43-59,
// 257-270, Maths.jl:299-328, 764-848), RamanPolarField with THG (Nonlinear.jl:282-333),
// the PreconStepper (RK45.jl:128-310, 343-406, dopri.jl:2-28) and Luna.run's stepfun and
// GridCondition saves (Luna.jl:358-391, Output.jl:490-502), on field-resolved grids and on
// envelope grids (Kerr_env, Nonlinear.jl:47-73; RamanPolarEnv, Nonlinear.jl:276-333; the
// two-sided padding of copy_scale_both!, NonlinearRHS.jl:56-114). It reads the same
// descriptors as the device library (include/luna_b200.h).
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <string>
#include <vector>

#include "../include/luna_b200.h"

typedef std::complex<double> cd;

namespace {

// ------------------------------------------------------------------ transforms
// Complex DFT of length M (power of two), iterative radix-2 decimation in time.
struct Fft {
    int M = 0;
    std::vector<cd> tw;  // exp(-2 pi i k / M), k < M/2
    std::vector<int> rev;
    void init(int m) {
        M = m;
        tw.resize(M / 2);
        for (int k = 0; k < M / 2; ++k) {
            const double a = -2.0 * M_PI * (double)k / (double)M;
            tw[k] = cd(std::cos(a), std::sin(a));
        }
        rev.assign(M, 0);
        int lg = 0;
        while ((1 << lg) < M) ++lg;
        for (int i = 0; i < M; ++i) {
            int r = 0;
            for (int b = 0; b < lg; ++b)
                if (i & (1 << b)) r |= 1 << (lg - 1 - b);
            rev[i] = r;
        }
    }
    // unnormalised: forward sum x e^{-2 pi i k n/M}, inverse with e^{+...}
    void run(cd* a, bool inv) const {
        for (int i = 0; i < M; ++i)
            if (i < rev[i]) std::swap(a[i], a[rev[i]]);
        for (int len = 2; len <= M; len <<= 1) {
            const int half = len / 2, step = M / len;
            for (int i = 0; i < M; i += len)
                for (int j = 0; j < half; ++j) {
                    cd w = tw[j * step];
                    if (inv) w = std::conj(w);
                    const cd u = a[i + j], v = a[i + j + half] * w;
                    a[i + j] = u + v;
                    a[i + j + half] = u - v;
                }
        }
    }
};

// Real DFT of even length n through one complex DFT of length n/2.
struct Rfft {
    int n = 0, M = 0;
    Fft f;
    std::vector<cd> W;  // exp(-2 pi i k / n), k <= M
    std::vector<cd> z;
    void init(int len) {
        n = len;
        M = n / 2;
        f.init(M);
        W.resize(M + 1);
        for (int k = 0; k <= M; ++k) {
            const double a = -2.0 * M_PI * (double)k / (double)n;
            W[k] = cd(std::cos(a), std::sin(a));
        }
        z.resize(M);
    }
    // X[k] = sum_t x[t] e^{-2 pi i k t/n}, k = 0..M
    void forward(const double* x, cd* X) {
        for (int m = 0; m < M; ++m) z[m] = cd(x[2 * m], x[2 * m + 1]);
        f.run(z.data(), false);
        X[0] = cd(z[0].real() + z[0].imag(), 0.0);
        X[M] = cd(z[0].real() - z[0].imag(), 0.0);
        for (int k = 1; k < M; ++k) {
            const cd Zk = z[k], Zm = std::conj(z[M - k]);
            X[k] = 0.5 * (Zk + Zm) - 0.5 * cd(0, 1) * W[k] * (Zk - Zm);
        }
    }
    // x[t] = sum_k X[k] e^{+2 pi i k t/n} over the Hermitian spectrum (unnormalised; the
    // imaginary parts of X[0] and X[M] are ignored, as irfft does)
    void inverse(const cd* X, double* x) {
        for (int k = 0; k < M; ++k) {
            cd Xk = X[k], Xm = X[M - k];
            if (k == 0) {
                Xk = cd(Xk.real(), 0.0);
                Xm = cd(Xm.real(), 0.0);
            }
            z[k] = (Xk + std::conj(Xm)) + cd(0, 1) * std::conj(W[k]) * (Xk - std::conj(Xm));
        }
        f.run(z.data(), true);
        for (int m = 0; m < M; ++m) {
            x[2 * m] = z[m].real();
            x[2 * m + 1] = z[m].imag();
        }
    }
};

// ------------------------------------------------------------------ plan
struct Resp {
    int kind = 0;
    double coef = 0, ionpot = 0, dt = 0, preion = 0, eratio = 0;
    std::vector<double> sx, sy, sD;
    double adk_pre = 0, adk_a = 0, adk_b = 0, adk_pw = 0, adk_thr = 0;
    std::vector<cd> H;  // rfft of the zero-padded Raman response (2 No points)
    double hdt = 0;
};

struct Plan {
    int kind = 0;  // 0: field-resolved, 1: envelope
    int N = 0, Nw = 0, No = 0;
    double in_scale = 0;
    std::vector<cd> outfac;
    std::vector<double> wwin, towin, twin;
    std::vector<Resp> resp;
    Rfft ro, rc, rr;
    Fft co, cc, cr;  // envelope grids: complex transforms of No, N and 2 No points
    bool raman = false;
    // scratch
    std::vector<cd> X, Xr;
    std::vector<cd> Ec, Pc, Rc;  // envelope fields
    std::vector<double> E, P, rate, frac, tmp, J, E2, pr;
    std::string err;
};

int fail(Plan* p, int code, const char* msg) {
    if (p) p->err = msg;
    return code;
}

// cumtrapz (Maths.jl:323-328): out[0] = 0, out[i] = out[i-1] + (y[i-1] + y[i])/2 dx
void cumtrapz(const double* y, double* out, int n, double dx) {
    double acc = 0.0;
    out[0] = 0.0;
    for (int i = 1; i < n; ++i) {
        acc += (0.5 * (y[i - 1] + y[i])) * dx;
        out[i] = acc;
    }
}

// PPT rate from the log-rate spline (Ionisation.jl:257-270, Maths.jl:772-774, 835-848);
// returns false above the table
bool ppt_rate(const Resp& r, double E, double* out) {
    const double aE = std::fabs(E);
    const int n = (int)r.sx.size();
    const double xmin = r.sx[0], xmax = r.sx[n - 1];
    if (aE > xmax) return false;
    if (!(aE >= xmin)) {  // below the table, or NaN (the numpy restatement masks both)
        *out = 0.0;
        return true;
    }
    int i1;
    if (aE <= xmin) i1 = 2;
    else if (aE >= xmax) i1 = n;
    else i1 = (int)std::ceil((aE - xmin) / (xmax - xmin) * (double)(n - 1)) + 1;
    i1 = std::max(2, std::min(n, i1));
    const int i = i1 - 1;
    const double xi = r.sx[i], xm = r.sx[i - 1], yi = r.sy[i], ym = r.sy[i - 1];
    double v;
    if (aE == xi) v = yi;
    else if (aE == xm) v = ym;
    else {
        const double Di = r.sD[i], Dm = r.sD[i - 1];
        const double t = (aE - xm) / (xi - xm);
        v = ym + Dm * t + (3 * (yi - ym) - 2 * Dm - Di) * (t * t) + (2 * (ym - yi) + Dm + Di) * (t * t * t);
    }
    *out = std::exp(v);
    return true;
}

// ADK rate (Ionisation.jl:43-59)
double adk_rate(const Resp& r, double E) {
    const double x = std::fabs(E);
    if (x < r.adk_thr || x == 0.0) return 0.0;
    return r.adk_pre * std::pow(r.adk_a / x, r.adk_pw) * std::exp(-r.adk_b / x);
}

// (t::TransModeAvg)(nl, Eω, z) on a field-resolved grid
int rhs(Plan* p, const cd* Ew, cd* nl) {
    const int No = p->No, M = No / 2;
    std::fill(p->X.begin(), p->X.end(), cd(0, 0));
    for (int k = 0; k < p->Nw && k <= M; ++k) p->X[k] = Ew[k];
    p->ro.inverse(p->X.data(), p->E.data());
    for (int t = 0; t < No; ++t) p->E[t] *= p->in_scale;
    std::fill(p->P.begin(), p->P.end(), 0.0);
    for (const Resp& r : p->resp) {
        if (r.kind == LUNA_RESP_KERR_FIELD) {
            for (int t = 0; t < No; ++t) {
                const double e = p->E[t];
                p->P[t] += r.coef * (e * e * e);
            }
        } else if (r.kind == LUNA_RESP_PLASMA_PPT || r.kind == LUNA_RESP_PLASMA_ADK) {
            for (int t = 0; t < No; ++t) {
                if (r.kind == LUNA_RESP_PLASMA_PPT) {
                    if (!ppt_rate(r, p->E[t], &p->rate[t]))
                        return fail(p, LUNA_FIELD_ABOVE_EMAX, "Field strength exceeds maximum for PPT ionisation rate.");
                } else {
                    p->rate[t] = adk_rate(r, p->E[t]);
                }
            }
            cumtrapz(p->rate.data(), p->frac.data(), No, r.dt);
            for (int t = 0; t < No; ++t) p->frac[t] = r.preion + 1 - std::exp(-p->frac[t]);
            for (int t = 0; t < No; ++t) p->tmp[t] = p->frac[t] * r.eratio * p->E[t];
            cumtrapz(p->tmp.data(), p->J.data(), No, r.dt);
            for (int t = 0; t < No; ++t)
                if (std::fabs(p->E[t]) > 0) p->J[t] += r.ionpot * p->rate[t] * (1 - p->frac[t]) / p->E[t];
            cumtrapz(p->J.data(), p->tmp.data(), No, r.dt);
            for (int t = 0; t < No; ++t) p->P[t] += r.coef * p->tmp[t];
        } else if (r.kind == LUNA_RESP_RAMAN) {
            std::fill(p->E2.begin(), p->E2.end(), 0.0);
            for (int t = 0; t < No; ++t) p->E2[t] = p->E[t] * p->E[t];
            p->rr.forward(p->E2.data(), p->Xr.data());
            for (int k = 0; k <= No; ++k) p->Xr[k] = r.H[k] * p->Xr[k] * r.hdt;
            p->rr.inverse(p->Xr.data(), p->pr.data());
            const double s = 1.0 / (2.0 * (double)No);
            for (int t = 0; t < No; ++t) p->P[t] += r.coef * p->E[t] * (p->pr[t] * s);
        } else {
            return fail(p, LUNA_ERR_UNSUPPORTED, "response not available in the CPU restatement");
        }
    }
    for (int t = 0; t < No; ++t) p->P[t] *= p->towin[t];
    p->ro.forward(p->P.data(), p->X.data());
    for (int k = 0; k < p->Nw; ++k) nl[k] = p->X[k] * p->outfac[k];
    return LUNA_OK;
}

// (t::TransModeAvg)(nl, Eω, z) on an envelope grid: the Nw bins go to both ends of the No
// bins (copy_scale_both!), complex transforms, the envelope responses
int rhs_env(Plan* p, const cd* Ew, cd* nl) {
    const int No = p->No, Nw = p->Nw, h = Nw / 2;
    std::fill(p->Ec.begin(), p->Ec.end(), cd(0, 0));
    for (int k = 0; k < h; ++k) p->Ec[k] = Ew[k];
    for (int j = 0; j < h; ++j) p->Ec[No - h + j] = Ew[Nw - h + j];
    p->co.run(p->Ec.data(), true);
    for (int t = 0; t < No; ++t) p->Ec[t] *= p->in_scale;
    std::fill(p->Pc.begin(), p->Pc.end(), cd(0, 0));
    for (const Resp& r : p->resp) {
        if (r.kind == LUNA_RESP_KERR_ENV) {
            for (int t = 0; t < No; ++t) {
                const cd e = p->Ec[t];
                p->Pc[t] += 3.0 / 4 * r.coef * std::norm(e) * e;
            }
        } else if (r.kind == LUNA_RESP_RAMAN) {
            std::fill(p->Rc.begin(), p->Rc.end(), cd(0, 0));
            for (int t = 0; t < No; ++t) p->Rc[t] = cd(0.5 * std::norm(p->Ec[t]), 0.0);
            p->cr.run(p->Rc.data(), false);
            for (int k = 0; k < 2 * No; ++k) p->Rc[k] = r.H[k] * p->Rc[k] * r.hdt;
            p->cr.run(p->Rc.data(), true);
            const double s = 1.0 / (2.0 * (double)No);
            for (int t = 0; t < No; ++t) p->Pc[t] += r.coef * p->Ec[t] * (p->Rc[t] * s);
        } else {
            return fail(p, LUNA_ERR_UNSUPPORTED, "response not available on envelope grids");
        }
    }
    for (int t = 0; t < No; ++t) p->Pc[t] *= p->towin[t];
    p->co.run(p->Pc.data(), false);
    if (Nw % 2) nl[h] = cd(0, 0);  // grids have even Nw; an odd middle bin has no source
    for (int k = 0; k < h; ++k) nl[k] = p->Pc[k] * p->outfac[k];
    for (int j = 0; j < h; ++j) nl[Nw - h + j] = p->Pc[No - h + j] * p->outfac[Nw - h + j];
    return LUNA_OK;
}

int rhs_any(Plan* p, const cd* Ew, cd* nl) { return p->kind == 0 ? rhs(p, Ew, nl) : rhs_env(p, Ew, nl); }

// ------------------------------------------------------------------ RK45 (dopri)
const double Bt[6][6] = {{1.0 / 5},
                         {3.0 / 40, 9.0 / 40},
                         {44.0 / 45, -56.0 / 15, 32.0 / 9},
                         {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729},
                         {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656},
                         {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84}};
const double NODES[6] = {1.0 / 5, 3.0 / 10, 4.0 / 5, 8.0 / 9, 1, 1};
const double B5[7] = {5179.0 / 57600, 0, 7571.0 / 16695, 393.0 / 640, -92097.0 / 339200, 187.0 / 2100, 1.0 / 40};
const double B4[7] = {35.0 / 384, 0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784, 11.0 / 84, 0};
const double IC[4][7] = {{1, 0, 0, 0, 0, 0, 0},
                         {-183.0 / 64, 0, 1500.0 / 371, -125.0 / 32, 9477.0 / 3392, -11.0 / 7, 3.0 / 2},
                         {37.0 / 12, 0, -1000.0 / 159, 125.0 / 12, -729.0 / 106, 11.0 / 3, -4},
                         {-145.0 / 128, 0, 1000.0 / 371, -375.0 / 64, 25515.0 / 6784, -55.0 / 28, 5.0 / 2}};

struct Stepper {
    Plan* p;
    int n;
    const cd* L;
    std::vector<cd> y, yn, tmp, out;
    std::vector<cd> ks[7];
    double t, tn, dt, dtn, rtol, atol, safety, max_dt, min_dt, err = 0, errlast = 0;
    bool ok = false;
    long long nrhs = 0;
    int status = LUNA_OK;

    void prop(std::vector<cd>& v, double d) {  // v *= exp(L d)
        for (int i = 0; i < n; ++i) v[i] *= std::exp(L[i] * d);
    }
    // make_fbar!: exp(-L d) f(exp(L d) ybar)
    void fbar(const std::vector<cd>& ybar, double t1, double t2, std::vector<cd>& res) {
        tmp = ybar;
        prop(tmp, t2 - t1);
        const int rc = rhs_any(p, tmp.data(), res.data());
        if (rc && status == LUNA_OK) status = rc;
        ++nrhs;
        prop(res, t1 - t2);
    }
    void evaluate() {
        y = yn;
        prop(ks[0], tn - t);
        dt = dtn;
        t = tn;
        std::vector<cd> st(n);
        for (int ii = 0; ii < 6; ++ii) {
            st = y;
            for (int jj = 0; jj <= ii; ++jj)
                if (Bt[ii][jj] != 0) {
                    const double c = dt * Bt[ii][jj];
                    for (int i = 0; i < n; ++i) st[i] = st[i] + c * ks[jj][i];
                }
            fbar(st, t, t + NODES[ii] * dt, ks[ii + 1]);
        }
    }
    void stepcontrol() {
        const double b1 = 3.0 / 5 / 5, b2 = -1.0 / 5 / 5, eps = 0.8;
        if (ok) {
            if (errlast == 0) errlast = err;
            const double fac = (err == 0) ? 1.5 : safety * std::pow(eps / err, b1) * std::pow(eps / errlast, b2);
            dtn = fac * dt;
            errlast = err;
        } else {
            dtn = std::isfinite(err) ? dt * std::max(0.1, safety * std::pow(err, -1.0 / 5)) : dt / 2;
        }
        if (dtn > max_dt) dtn = max_dt;
        else if (dtn < min_dt) {
            dtn = min_dt;
            ok = true;
        }
    }
    // replay (verification aid, as in the device solver): the accept decision and the next
    // step size come from a recorded sequence instead of the controller
    const double* replay = nullptr;
    long long nreplay = 0, nstep = 0;
    bool step() {
        evaluate();
        std::vector<cd> nn = y;
        for (int jj = 0; jj < 7; ++jj)
            if (B5[jj] != 0) {
                const double c = dt * B5[jj];
                for (int i = 0; i < n; ++i) nn[i] = nn[i] + c * ks[jj][i];
            }
        yn = nn;
        std::vector<cd> ye(n, cd(0, 0));
        for (int ii = 0; ii < 7; ++ii) {
            const double e = B5[ii] - B4[ii];
            if (e != 0)
                for (int i = 0; i < n; ++i) ye[i] = ye[i] + dt * ks[ii][i] * e;
        }
        double sy = 0, syn = 0, se = 0;
        for (int i = 0; i < n; ++i) {
            sy += std::norm(y[i]);
            syn += std::norm(yn[i]);
            se += std::norm(ye[i]);
        }
        const double errwt = std::max(std::max(std::sqrt(sy), std::sqrt(syn)), atol);
        err = std::sqrt(se) / rtol / errwt;
        ok = err <= 1;
        stepcontrol();
        if (replay && nstep < nreplay) {
            ok = replay[2 * nstep + 1] != 0.0;
            if (nstep + 1 < nreplay) dtn = replay[2 * (nstep + 1)];
        }
        ++nstep;
        if (ok) {
            tn = t + dt;
            ks[0] = ks[6];
        } else {
            yn = y;
        }
        prop(yn, tn - t);
        return ok;
    }
    void interpolate(double ti, cd* o) {
        if (ti == t) {
            std::copy(y.begin(), y.end(), o);
            return;
        }
        if (ti == tn) {
            std::copy(yn.begin(), yn.end(), o);
            return;
        }
        const double s = (ti - t) / dt;
        const double sp[4] = {s, s * s, s * s * s, (s * s) * (s * s)};
        double b[7];
        for (int j = 0; j < 7; ++j) {
            b[j] = 0;
            for (int q = 0; q < 4; ++q) b[j] += sp[q] * IC[q][j];
        }
        for (int i = 0; i < n; ++i) {
            cd yi(0, 0);
            for (int j = 0; j < 7; ++j) yi = yi + ks[j][i] * b[j];
            o[i] = (y[i] + dt * yi) * std::exp(L[i] * (ti - t));
        }
    }
};

}  // namespace

extern "C" {

int uo_plan_create(const luna_grid_desc* g, const luna_resp_desc* rs, int nresp, void** out) {
    if (!g || !out || (nresp > 0 && !rs)) return LUNA_ERR_BAD_ARG;
    if (g->kind != 0 && g->kind != 1) return LUNA_ERR_UNSUPPORTED;
    Plan* p = new Plan();
    p->kind = g->kind;
    p->N = g->N;
    p->Nw = g->Nw;
    p->No = g->No;
    p->in_scale = g->in_scale;
    p->outfac.resize(g->Nw);
    for (int k = 0; k < g->Nw; ++k) p->outfac[k] = cd(g->outfac[2 * k], g->outfac[2 * k + 1]);
    p->wwin.assign(g->wwin, g->wwin + g->Nw);
    p->towin.assign(g->towin, g->towin + g->No);
    p->twin.assign(g->twin, g->twin + g->N);
    const bool env = g->kind == 1;
    if (env) {
        p->co.init(g->No);
        p->cc.init(g->N);
    } else {
        p->ro.init(g->No);
        p->rc.init(g->N);
    }
    const int No = g->No;
    for (int i = 0; i < nresp; ++i) {
        const luna_resp_desc& d = rs[i];
        Resp r;
        r.kind = d.kind;
        r.coef = d.coef;
        if (d.kind == LUNA_RESP_PLASMA_PPT || d.kind == LUNA_RESP_PLASMA_ADK) {
            r.ionpot = d.ionpot;
            r.dt = d.dt;
            r.preion = d.preionfrac;
            r.eratio = d.eratio;
            if (d.kind == LUNA_RESP_PLASMA_PPT) {
                r.sx.assign(d.spl_x, d.spl_x + d.spl_n);
                r.sy.assign(d.spl_y, d.spl_y + d.spl_n);
                r.sD.assign(d.spl_D, d.spl_D + d.spl_n);
            }
            r.adk_pre = d.adk_pre;
            r.adk_a = d.adk_a;
            r.adk_b = d.adk_b;
            r.adk_pw = d.adk_pw;
            r.adk_thr = d.adk_thr;
        } else if (d.kind == LUNA_RESP_RAMAN) {
            // h(t) = sum_i hpre_i(t) exp(-t/tau2_i) w(t) on the first half of 2 No points
            // (CombinedRamanResponse, Raman.jl:249-262), then its real spectrum
            if (!p->raman) {
                if (env) p->cr.init(2 * No);
                else p->rr.init(2 * No);
                p->raman = true;
            }
            std::vector<double> h(2 * No, 0.0);
            for (int t = 0; t < No; ++t) {
                double acc = 0;
                for (int c = 0; c < d.ncomp; ++c) acc += d.hpre[(size_t)c * No + t] * std::exp(-d.htt[t] / d.tau2[c]);
                h[t] = acc * d.hwin[t];
            }
            if (env) {  // complex spectrum of the 2 No-point response (RamanPolarEnv)
                r.H.assign(2 * No, cd(0, 0));
                for (int t = 0; t < 2 * No; ++t) r.H[t] = cd(h[t], 0.0);
                p->cr.run(r.H.data(), false);
            } else {
                r.H.resize(No + 1);
                p->rr.forward(h.data(), r.H.data());
            }
            r.hdt = d.hdt;
        } else if (d.kind != (env ? LUNA_RESP_KERR_ENV : LUNA_RESP_KERR_FIELD)) {
            delete p;
            return LUNA_ERR_UNSUPPORTED;
        }
        p->resp.push_back(r);
    }
    p->X.resize(No / 2 + 1);
    p->Xr.resize(No + 1);
    p->E.resize(No);
    p->P.resize(No);
    p->rate.resize(No);
    p->frac.resize(No);
    p->tmp.resize(No);
    p->J.resize(No);
    p->E2.resize(2 * No);
    p->pr.resize(2 * No);
    if (env) {
        p->Ec.resize(No);
        p->Pc.resize(No);
        p->Rc.resize(2 * No);
    }
    *out = p;
    return LUNA_OK;
}

void uo_plan_destroy(void* h) { delete static_cast<Plan*>(h); }

int uo_rhs(void* h, double* nl, const double* Ew) {
    Plan* p = static_cast<Plan*>(h);
    return rhs_any(p, reinterpret_cast<const cd*>(Ew), reinterpret_cast<cd*>(nl));
}

// Luna.run with RK45.solve_precon (a MemoryOutput on saveN GridCondition points): y_inout
// holds Eω on entry and the final state on return; saves [saveN][Nw] complex; steplog
// (optional) [4*o->steplog_cap] rows (z, dz, err, accepted) of the first steps, the rows of
// the device solver's step log.
int uo_solve(void* h, const double* linop, double* y_inout, double z0, double dz0, double zmax,
             const luna_solve_opts* o, double* saves, double* steplog, luna_solve_stats* stats) {
    Plan* p = static_cast<Plan*>(h);
    const int n = p->Nw;
    Stepper s;
    s.p = p;
    s.n = n;
    s.L = reinterpret_cast<const cd*>(linop);
    s.y.assign(reinterpret_cast<cd*>(y_inout), reinterpret_cast<cd*>(y_inout) + n);
    s.yn = s.y;
    s.tmp.resize(n);
    for (int j = 0; j < 7; ++j) s.ks[j].assign(n, cd(0, 0));
    s.t = s.tn = z0;
    s.dt = s.dtn = dz0;
    s.rtol = o->rtol;
    s.atol = o->atol;
    s.safety = o->safety;
    s.max_dt = o->max_dt;
    s.min_dt = o->min_dt;
    s.replay = o->replay;
    s.nreplay = o->replay ? o->nreplay : 0;
    s.fbar(s.y, s.t, s.t, s.ks[0]);
    int saved = 0, repeated = 0;
    long long steps = 0, rejected = 0;
    int status = s.status;
    std::vector<double> Et(p->N);
    std::vector<cd> Y(p->N / 2 + 1), Yc(p->kind == 1 ? p->N : 0);
    cd* sv = reinterpret_cast<cd*>(saves);
    while (status == LUNA_OK && s.tn <= zmax) {
        const double zstep = s.tn, dzstep = s.dtn;  // the step about to be taken (evaluate())
        const bool ok = s.step();
        if (steplog && steps < o->steplog_cap) {
            double* row = steplog + 4 * steps;
            row[0] = zstep;
            row[1] = dzstep;
            row[2] = s.err;
            row[3] = ok ? 1.0 : 0.0;
        }
        ++steps;
        if (s.status != LUNA_OK) {
            status = s.status;
            break;
        }
        if (ok) {
            // stepfun (Luna.jl:366-372): ωwin, back to time, twin, forward
            if (p->kind == 0) {
                for (int k = 0; k < n; ++k) Y[k] = s.yn[k] * p->wwin[k];
                for (int k = n; k <= p->N / 2; ++k) Y[k] = cd(0, 0);
                p->rc.inverse(Y.data(), Et.data());
                for (int t = 0; t < p->N; ++t) Et[t] = Et[t] / (double)p->N * p->twin[t];
                p->rc.forward(Et.data(), Y.data());
                for (int k = 0; k < n; ++k) s.yn[k] = Y[k];
            } else {
                for (int k = 0; k < n; ++k) Yc[k] = s.yn[k] * p->wwin[k];
                p->cc.run(Yc.data(), true);
                for (int t = 0; t < p->N; ++t) Yc[t] = Yc[t] / (double)p->N * p->twin[t];
                p->cc.run(Yc.data(), false);
                for (int k = 0; k < n; ++k) s.yn[k] = Yc[k];
            }
            while (saved < o->saveN && o->zsave[saved] <= s.tn) {
                if (sv) s.interpolate(o->zsave[saved], sv + (size_t)saved * n);
                ++saved;
            }
            repeated = 0;
        } else {
            ++rejected;
            if (++repeated > o->repeat_limit) {
                status = LUNA_REPEAT_LIMIT;
                break;
            }
        }
        if (o->max_steps > 0 && steps >= o->max_steps) {
            if (s.tn <= zmax) status = LUNA_STEP_BUDGET;
            break;
        }
    }
    std::copy(s.yn.begin(), s.yn.end(), reinterpret_cast<cd*>(y_inout));
    if (stats) {
        std::memset(stats, 0, sizeof(*stats));
        stats->status = status;
        stats->nsaved = saved;
        stats->steps = steps;
        stats->accepted = steps - rejected;
        stats->rejected = rejected;
        stats->nrhs = s.nrhs;
        stats->z = s.tn;
        stats->dz = s.dtn;
    }
    return status;
}

const char* uo_last_error(void* h) { return h ? static_cast<Plan*>(h)->err.c_str() : ""; }

}  // extern "C"
