// Device-visible description of one propagation instance (plan + solver state).
// Filled by the host side of the C ABI; read by the persistent solver kernel.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define LUNA_MAX_RESP 4
#ifndef LUNA_NSTATS
#define LUNA_NSTATS 10
#endif

// response kinds (same values as the public header)
#ifndef LUNA_RESP_KERR_FIELD
#define LUNA_RESP_KERR_FIELD 1
#define LUNA_RESP_KERR_ENV 2
#define LUNA_RESP_PLASMA_PPT 3
#define LUNA_RESP_PLASMA_ADK 4
#define LUNA_RESP_RAMAN 5
#endif

typedef struct {
    int kind;
    double coef;      // Kerr: rho*eps0*gamma3; Raman: rho; plasma: rho
    // plasma (PlasmaCumtrapz)
    double ionpot, dt, preion, eratio;
    // PPT log-rate spline on a uniform field axis
    const double* sx;
    const double* sy;
    const double* sD;
    const float* sxf;
    const float* syf;
    const float* sDf;
    int sn;
    double Emin, Emax;
    // ADK: rate = pre * (a/|E|)^pw * exp(-b/|E|) for |E| >= thr
    double adk_pre, adk_a, adk_b, adk_pw, adk_thr;
    // Raman: spectrum H[k], k = 0..No, of the normalised response on the 2*No grid
    // (complex of the compute precision); coef carries rho * max|h| * dt / (2*No)
    const void* H;
    // Raman response build inputs (used once at plan creation)
    const double* hpre;    // [ncomp * No] undamped responses
    const double* tau2;    // [ncomp] dephasing times at this density
    const double* hwin;    // [No] window
    const double* htt;     // [No] response time axis
    double hdt;            // response grid spacing
    int ncomp;
    // no-THG forms (Kerr_field_nothg, RamanPolarField(thg=false)): the squared field is
    // |hilbert(E)|^2 = E^2 + H^2, H the Hilbert transform of E (kind stays KERR_FIELD /
    // RAMAN)
    int hilb;
    // Kerr_env_thg (kind KERR_ENV): [No] exp(2i w0 t) on the oversampled grid, or null
    const double2* cthg;
    // Raman with a pressure gradient: [4 * ncomp] (model, A, B, C) of tau2(rho) per
    // component, or null; amg the amagat density; hscale = 1/max|hpre| (the normalisation of
    // the spectrum); hz = 1 when H is rebuilt at rho(z) in place (read with plain loads)
    const double* t2rho;
    double amg, hscale;
    int hz;
} LunaResp;
#define LUNA_RAMAN_MAXC 4  // components of a density-dependent Raman response

// Pressure-gradient fill and/or taper (z-dependent density, radius, normalisation and
// linear operator); the fields mirror luna_gradient_desc of the public header.
#define LUNA_GRAD_NPTS 16
typedef struct {
    int npts, two_point, loss, nta;
    double Z[LUNA_GRAD_NPTS], P[LUNA_GRAD_NPTS], P2[LUNA_GRAD_NPTS];
    double ZA[LUNA_GRAD_NPTS], A[LUNA_GRAD_NPTS];
    double dens_a, dens_b, unm, aeff_intg, in_base, eps0c2;
    const double* gam;    // [Nw]
    const double2* vn;    // [Nw]
    const double* wc;     // [Nw] ω/c on sidx, 0 elsewhere
    const double* om;     // [Nw]
    const double* imcap;  // [Nw]
    const double2* ofs;   // [Nw]
    double fd_xc[4], fd_gam[4];
    double2 fd_vn[4];
    double fd_h12;
    // envelope grid without THG: + i β(ω0; z), β from neff at ω0 (ω0/c, γ(ω0), vn(ω0))
    int bref;
    double ref_xc, ref_gam;
    double2 ref_vn;
} LunaGrad;

typedef struct {
    // ---- grid / transform (NonlinearRHS.TransModeAvg) ----
    int kind;            // 0: field-resolved (RealGrid), 1: envelope (EnvGrid)
    int N, Nw, No;       // coarse time samples, coarse frequency bins, oversampled samples
    const double2* linop;   // [Nw]
    const double2* outfac;  // [Nw] crop scale x (norm * sqrt(Aeff) * omega window on sidx, 1 elsewhere)
    const double* wwin;     // [Nw] omega window (stepfun)
    const double* towin;    // [No]
    const double* twin;     // [N] (stepfun)
    double in_scale;        // pad scale / No / (nlscale * sqrt(Aeff))
    const double* omega;    // [Nw] grid.ω (per-step statistics; may be null)
    const double* tgrid;    // [N] grid.t (per-step statistics)
    double aeff;            // effective area (per-step statistics)
    double escale;          // 1/sqrt(eps0*c*Aeff/2): mode-averaged field -> V/m
    int nresp;
    LunaResp resp[LUNA_MAX_RESP];
    // pressure gradient / taper (null: constant density, area and linop); linz/outz hold
    // L(z) and the output factor at the current stage node, written by the solver;
    // outz[Nw] = (field scale, Aeff) at that node
    const LunaGrad* grad;
    double2* linz;  // [Nw]
    double2* outz;  // [Nw + 1]
    int ramz;       // 1 + index of a Raman response rebuilt at rho(z) (its H is writable), 0: none
    // ---- integrator (RK45.solve_precon) ----
    const double2* y0;   // [Nw] initial field (kept, so a batch can be re-run)
    double2* y;
    double2* yn;
    void* k[7];          // stage derivatives, double2 (plain) or float2 (mixed)
    double2* e1;         // exp(L*dz) of the last stage-5 node
    void* gscr;          // global scratch for buffers that do not fit in shared memory
    double2* saves;      // [saveN * Nw]
    const double* zsave; // [saveN]
    int saveN;
    double z0, dz0, zmax, rtol, atol, safety, max_dt, min_dt;
    int repeat_limit;
    long long max_steps;
    double* steplog;     // optional [4 * steplog_cap]: t, dt, err, ok per step
    long long steplog_cap;
    const double* replay; // optional [2 * nreplay]: (dt, ok) of each step to follow
    long long nreplay;
    double* stats;        // optional [LUNA_NSTATS * stats_cap]: Stats.default row per accepted step
    long long stats_cap;
    long long nstats;
    // ---- results ----
    int status;
    int nsaved;
    long long steps, accepted, rejected, nrhs;
    double z, dz;
    unsigned long long t_begin, t_end;  // device global timer (ns) around the integration
    int sm;                             // SM that integrated the instance
} LunaInst;
