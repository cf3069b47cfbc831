/*
 * libluna_b200 — C ABI of the B200 (sm_100a) UPPE right-hand side and RK45 integrator.
 *
 * This library replaces, for one GPU, the hot path of Luna.jl v0.6.2:
 *   - the mode-averaged transform  (t::TransModeAvg)(nl, Eω, z)   NonlinearRHS.jl:362-373
 *     with its responses  Kerr_field / Kerr_env                   Nonlinear.jl:8-73
 *                         PlasmaCumtrapz (PPT spline / ADK rate)  Nonlinear.jl:88-177,
 *                                                                 Ionisation.jl:22-63, 247-271
 *                         RamanPolarField / RamanPolarEnv         Nonlinear.jl:183-333,
 *                                                                 Raman.jl:242-262
 *   - the integrator RK45.solve_precon(...) and Luna.run's loop    RK45.jl:19-89, 128-406,
 *     (window filter stepfun, GridCondition saves)                Luna.jl:358-391,
 *                                                                 Output.jl:65-82, 490-502
 *
 * Conventions
 *   - Complex arrays are interleaved (re, im) doubles, i.e. the memory layout of Julia's
 *     Vector{ComplexF64}; `Nw` complex values = 2*Nw doubles.
 *   - Every entry point returns a status code (LUNA_OK = 0 on success); the message of the
 *     last failure on the calling thread is available from luna_b200_last_error().
 *   - A plan owns its device copies of the grid, normalisation and response tables. Calls
 *     on one plan must be serialised; different plans may be used from different threads.
 *   - There is no CPU fallback: without a usable CUDA device every call fails with
 *     LUNA_ERR_CUDA.
 *   - The library keeps per-device state for the life of the process (twiddle tables, the
 *     device address of the allocation-free entry point's buffer). Destroying a device's
 *     primary context (cudaDeviceReset) invalidates it together with every plan and batch
 *     on that device: do not call the library on that device again in the same process.
 */
#ifndef LUNA_B200_H
#define LUNA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define LUNA_OK 0
#define LUNA_FIELD_ABOVE_EMAX 1 /* PPT field above the table maximum (Ionisation.jl:262-265) */
#define LUNA_REPEAT_LIMIT 2     /* more than repeat_limit rejected steps (RK45.jl:72-76) */
#define LUNA_NONFINITE 3
#define LUNA_STEP_BUDGET 4      /* max_steps reached before zmax */
#define LUNA_WAIT_TIMEOUT 5     /* a bounded device-side wait gave up (the result is invalid) */
#define LUNA_ERR_BAD_ARG 16
#define LUNA_ERR_UNSUPPORTED 17
#define LUNA_ERR_CUDA 18

/* response kinds */
#define LUNA_RESP_KERR_FIELD 1  /* Nonlinear.Kerr_field(γ3)                 Nonlinear.jl:24-34 */
#define LUNA_RESP_KERR_ENV 2    /* Nonlinear.Kerr_env(γ3)                   Nonlinear.jl:63-73 */
#define LUNA_RESP_PLASMA_PPT 3  /* PlasmaCumtrapz with ionrate_fun!_PPTcached  Nonlinear.jl:107 */
#define LUNA_RESP_PLASMA_ADK 4  /* PlasmaCumtrapz with ionrate_fun!_ADK         Nonlinear.jl:107 */
#define LUNA_RESP_RAMAN 5       /* RamanPolarField(thg=true) / RamanPolarEnv Nonlinear.jl:223-264 */
#define LUNA_RESP_KERR_FIELD_NOTHG 6 /* Nonlinear.Kerr_field_nothg(γ3, n): 3/4 ρ ε0 γ3 |hilbert(E)|^2 E
                                        Nonlinear.jl:36-45 (RealGrid)                     */
#define LUNA_RESP_RAMAN_NOTHG 7 /* RamanPolarField(t, r; thg=false): the convolution of
                                   1/2 |hilbert(E)|^2 (sqr!, Nonlinear.jl:267-275); fields as
                                   LUNA_RESP_RAMAN (RealGrid)                              */
#define LUNA_RESP_KERR_ENV_THG 8 /* Nonlinear.Kerr_env_thg(γ3, ω0, t): ρ ε0 γ3/4 (3|E|^2 +
                                    exp(2iω0t) E^2) E, Nonlinear.jl:75-84 (EnvGrid); coef and
                                    cthg                                                   */

/* precision modes */
#define LUNA_PREC_FP64 0  /* plain: every operation in FP64 */
#define LUNA_PREC_MIXED 1 /* FP32 transforms/responses/stage derivatives; FP64 state, phase,
                             controller, norms and plasma prefix sums */

/* Grid and normalisation of one TransModeAvg (Grid.jl:12-194, NonlinearRHS.jl:375-399). */
typedef struct {
    int kind;              /* 0: RealGrid (field-resolved), 1: EnvGrid (envelope)        */
    int N;                 /* coarse time samples length(grid.t)                         */
    int Nw;                /* coarse frequency bins length(grid.ω)                       */
    int No;                /* oversampled time samples length(grid.to)                   */
    const double* outfac;  /* [2*Nw] crop scale x (norm*sqrt(Aeff)*ωwin on sidx, 1 else) */
    const double* wwin;    /* [Nw] grid.ωwin                                             */
    const double* towin;   /* [No] grid.towin                                            */
    const double* twin;    /* [N]  grid.twin                                             */
    double in_scale;       /* pad scale / No / (nlscale*sqrt(Aeff))                      */
    /* per-step statistics (Stats.default); may be NULL / 0 when they are not requested */
    const double* omega;   /* [Nw] grid.ω                                                */
    const double* t;       /* [N]  grid.t                                                */
    double aeff;           /* effective area Aeff                                        */
    double escale;         /* 1/sqrt(ε0 c Aeff/2): mode-averaged field to V/m            */
} luna_grid_desc;

/* One nonlinear response, applied in the order given (Et_to_Pt!, NonlinearRHS.jl:121-126). */
typedef struct {
    int kind;               /* LUNA_RESP_*                                               */
    double coef;            /* Kerr: ρ*ε0*γ3; plasma and Raman: ρ                         */
    /* PlasmaCumtrapz */
    double ionpot;          /* ionisation potential [J]                                  */
    double dt;              /* t[2]-t[1] of the oversampled grid                         */
    double preionfrac;      /* in [0, 1]                                                 */
    double eratio;          /* e^2/m_e                                                   */
    const double* spl_x;    /* [spl_n] uniform field axis of the PPT log-rate spline     */
    const double* spl_y;    /* [spl_n] log(rate)                                         */
    const double* spl_D;    /* [spl_n] Hermite slopes (Maths.jl:812-828)                 */
    int spl_n;
    double adk_pre, adk_a, adk_b, adk_pw, adk_thr; /* rate = pre*(a/|E|)^pw*exp(-b/|E|)   */
    /* Raman (CombinedRamanResponse evaluated at the plan's density) */
    int ncomp;
    const double* hpre;     /* [ncomp*No] undamped component responses on htt             */
    const double* tau2;     /* [ncomp] dephasing time of each component at this density  */
    const double* hwin;     /* [No] Planck-taper window of the response                  */
    const double* htt;      /* [No] response time axis (0..No-1)*dt                      */
    double hdt;             /* response grid spacing (scales the convolution)            */
    /* Kerr_env_thg */
    const double* cthg;     /* [2*No] exp(2iω0 t) on the oversampled grid.to (complex)   */
    /* Raman with a pressure gradient: the density dependence of each component's
     * dephasing time, [4*ncomp] rows (model, A, B, C), or NULL when no component depends on
     * the density. model 0: tau2[c] at every density; model 1 (RamanRespRotationalNonRigid
     * with Bρ, Raman.jl:229-238): τ2(ρ) = 1/(π (A/(ρ/amg) + B ρ/amg)) for ρ > 0, ∞ at ρ = 0;
     * model 2 (RamanRespVibrational with Bρ, Raman.jl:142-157): τ2(ρ) = 1/(π (C + A/(ρ/amg)
     * + B ρ/amg)). Used only once a gradient is attached: the response spectrum is then
     * rebuilt at ρ(z) of every stage node, as the reference rebuilds h(t; ρ) at every call
     * (Nonlinear.jl:306-307). */
    const double* tau2_rho;
    double amg;             /* the amagat density [m^-3] of the τ2(ρ) laws                */
} luna_resp_desc;

typedef struct {
    double rtol, atol, safety, max_dt, min_dt; /* RK45.solve_precon keywords (RK45.jl:19-21) */
    int repeat_limit;                          /* RK45.solve keyword (RK45.jl:27-28)        */
    long long max_steps;                       /* 0: unlimited                              */
    int saveN;                                 /* number of GridCondition save points       */
    const double* zsave;                       /* [saveN] save points (Output.jl:495-497)   */
    long long steplog_cap;                     /* rows of (z, dz, err, ok) to record; 0: off */
    const double* replay;                      /* optional [2*nreplay] (dz, accepted) per step:
                                                  follow this step sequence instead of the
                                                  controller's choice (verification aid)      */
    long long nreplay;
    int flags;                                 /* LUNA_SOLVE_* bits, 0 for the defaults     */
    long long stats_cap;                       /* rows of per-step statistics; 0: off       */
    int dist_min_no;                           /* batches: instances with at least this many
                                                  oversampled samples run on a cluster of CTAs
                                                  each (in the batch's precision); 0: 16384  */
} luna_solve_opts;

/* Per-step statistics (Stats.default, Stats.jl:495-532, for a mode-averaged field-resolved
 * transform), one row of LUNA_NSTATS doubles per accepted step, in this order:
 * z, dz, ω0, energy, peakpower, peakintensity, fwhm_t_min, fwhm_t_max, electrondensity,
 * peak_ionisation_rate (the last two NaN without a plasma response). */
#define LUNA_NSTATS 10

/* luna_solve_opts.flags */
#define LUNA_SOLVE_NO_DIST 2     /* batches: no distributed (multi-CTA) integration of the
                                    long instances; a verification and timing aid          */
#define LUNA_SOLVE_NO_CLUSTERS 1 /* batches: integrate every instance on one CTA (no Raman
                                    clusters, no distributed instances); a verification
                                    and timing aid                                      */

typedef struct {
    int status;
    int nsaved;
    long long steps, accepted, rejected, nrhs;
    double z, dz; /* final z (first tn > zmax) and next step size */
    long long nstats; /* rows of per-step statistics recorded */
} luna_solve_stats;

typedef struct luna_plan luna_plan;
typedef struct luna_batch luna_batch;

/* Replaces the TransModeAvg constructor (NonlinearRHS.jl:344-358) as built by Luna.setup
 * (Luna.jl:115-151): copies grid, normalisation and response tables to the device. */
int luna_b200_plan_create(const luna_grid_desc* grid, const luna_resp_desc* resps, int nresp,
                          int precision, luna_plan** out);
void luna_b200_plan_destroy(luna_plan* plan);

/* (t::TransModeAvg)(nl, Eω, z)  — NonlinearRHS.jl:362-373. Host arrays of Nw complex. */
int luna_b200_rhs(luna_plan* plan, double* nl, const double* Ew, double z);
/* Same with device pointers, enqueued on `stream` (a cudaStream_t, may be NULL). */
int luna_b200_rhs_device(luna_plan* plan, double* nl_dev, const double* Ew_dev, double z, void* stream);

/* ---------------------------------------------------------------- pressure gradients, tapers
 * A gas fill whose pressure varies along the fibre, Capillary.gradient(gas, L, p0, p1) or
 * Capillary.gradient(gas, Z, P) (Capillary.jl:306-337), and/or a core radius a(z)
 * (MarcatiliMode(afun, ...), Interface.jl:249-250), in a MarcatiliMode of the full model.
 * Attached to a plan it makes the transform z-dependent, as TransModeAvg is with a density
 * function, aeff(z) and βfun!(β, z) (NonlinearRHS.jl:362-387): the response coefficients
 * are given for ρ = 1 and the polarisation is scaled by ρ(z); the field scale is
 * in_base/sqrt(Aeff(z)) and the normalisation on sidx pre sqrt(Aeff(z))/β(z). The solvers
 * evaluate the linear operator of LinearOps.make_linop (LinearOps.jl:330-360) at every
 * stage node, save point and step end (make_prop! for a z-dependent linop, RK45.jl:284-297):
 *   p(z) = sqrt(P[i]^2 + (z - Z[i])/(Z[i+1] - Z[i]) (P[i+1]^2 - P[i]^2)) on segment i,
 *   ρ(z) = dens_a p / (1 + dens_b p),  coren = sqrt(1 + γ(ω) ρ),
 *   a(z) = A[i] + (z - ZA[i])/(ZA[i+1] - ZA[i]) (A[i+1] - A[i]) (A[0] / A[end] outside),
 *   nwg = (unm/(k a))^2 (1 - i vn/(k a))^2,  neff = sqrt(coren^2 - nwg) (principal root),
 *   β1(z) = (-f(ω0+2h) + 8 f(ω0+h) - 8 f(ω0-h) + f(ω0-2h)) / (12 h), f(x) = x/c Re neff(x)
 *           with Re neff raised to 1e-3 where it is below (Capillary.jl:162-173),
 *   L(ω; z) = -i (ω/c conj_clamp(neff) - ω β1(z)) on sidx, 0 elsewhere (LinearOps.jl:254),
 *   β(ω; z) = ω/c Re neff (with the 1e-3 rule when the radius has more than one node),
 *   Aeff(z) = a(z)^2 aeff_intg (Capillary.jl:295),
 * each in IEEE-rounded real operations in the order written (no fused multiply-adds).
 * The linop argument of the solve entry points is ignored for such a plan (may be NULL).
 * Field-resolved and envelope grids (for the latter see env_ref). A Raman response whose dephasing times depend on the density
 * (luna_resp_desc.tau2_rho) has its spectrum rebuilt at ρ(z) before every evaluation (one
 * extra transform of the 2*No response grid); its rebuild buffer is per plan for the RHS
 * entry points and per instance in a batch. */
#define LUNA_GRAD_MAXPTS 16
typedef struct {
    int npts;                    /* pressure nodes, 2..LUNA_GRAD_MAXPTS                     */
    int two_point;               /* 1: gradient(gas, L, p0, p1): P[0] for z <= 0, P[1] for
                                    z > L; 0: (Z, P) form: P[0] for z <= Z[0], P[end] for
                                    z >= Z[end]                                              */
    double Z[LUNA_GRAD_MAXPTS];  /* node positions, increasing (two-point: 0, L)            */
    double P[LUNA_GRAD_MAXPTS];  /* node pressures [bar]; equal values: constant pressure   */
    double P2[LUNA_GRAD_MAXPTS]; /* P[i]*P[i]                                               */
    double dens_a, dens_b;       /* ρ(p) = dens_a p / (1 + dens_b p) [m^-3], p in bar        */
    int loss;                    /* 0: real effective index (MarcatiliMode loss=false)      */
    int nta;                     /* radius nodes, 1 (constant radius)..LUNA_GRAD_MAXPTS     */
    double ZA[LUNA_GRAD_MAXPTS]; /* radius node positions, increasing                       */
    double A[LUNA_GRAD_MAXPTS];  /* core radius at the nodes [m]                            */
    double unm;                  /* mode's Bessel zero                                      */
    double aeff_intg;            /* Aeff / a^2                                              */
    double in_base;              /* pad scale / No / nlscale                                */
    double eps0c2;               /* ε0 c / 2 (field scale of the statistics)                */
    const double* gam;           /* [Nw] γ(ω): Sellmeier susceptibility per unit density    */
    const double* vn;            /* [2*Nw] cladding term get_vn(εcl(ω)) (Capillary.jl:88-93) */
    const double* wc;            /* [Nw] ω/c on sidx, 0 elsewhere                           */
    const double* om;            /* [Nw] ω (ω - ω0 on an envelope grid)                     */
    const double* imcap;         /* [Nw] 3000 c/ω: conj_clamp's bound on Im neff            */
    const double* ofs;           /* [2*Nw] crop scale x pre*ωwin on sidx (times
                                    sqrt(Aeff(z))/β(z) on the device), crop scale else;
                                    pre = -i ω^2/(4 nlscale c)                              */
    double fd_xc[4];             /* x/c at x = ω0+2h, ω0+h, ω0-h, ω0-2h (h = 1e-4 ω0)        */
    double fd_gam[4];            /* γ(x)                                                    */
    double fd_vn[8];             /* vn(x), complex                                          */
    double fd_h12;               /* 12 h                                                    */
    /* envelope grids (kind 1; om above holds ω - ω0): make_linop for EnvGrid
     * (LinearOps.jl:363-388) adds + i β(ω0; z) without THG, β(ω0; z) = ω0/c Re neff(ω0; z)
     * (the 1e-3 rule with more than one radius node) */
    int env_ref;                 /* 1: take out β(ω0; z) (thg = false), 0: thg = true        */
    double ref_xc;               /* ω0/c                                                    */
    double ref_gam;              /* γ(ω0)                                                   */
    double ref_vn[2];            /* vn(ω0), complex                                         */
} luna_gradient_desc;
/* Attach (or, with grad == NULL, remove) a pressure gradient and/or taper. Replaces building
 * the transform with densityfun/aeff/βfun! and the linop with make_linop (Luna.jl:115-151). */
int luna_b200_plan_set_gradient(luna_plan* plan, const luna_gradient_desc* grad);
/* linop!(out, z) of make_linop (LinearOps.jl:330-360) for a plan with a pressure gradient
 * or taper, evaluated on the device as the solvers do: linop [2*Nw] receives L(ω; z);
 * outfac (optional, [2*Nw]) the output factor ρ(z) x crop scale x pre*sqrt(Aeff(z))*ωwin/β(z)
 * (ρ(z) x crop scale off sidx). Host arrays. */
int luna_b200_plan_linop(luna_plan* plan, double z, double* linop, double* outfac);

/* RK45.solve_precon(transform, linop, Eω, z0, dz0, zmax; ...) driven by Luna.run
 * (Luna.jl:358-391): integrates y_inout in place to the first step beyond zmax, saving the
 * GridCondition points into `saves` ([saveN*2*Nw] doubles) and optionally the step log
 * ([4*steplog_cap] doubles). All pointers are host memory. */
int luna_b200_solve(luna_plan* plan, const double* linop, double* y_inout, double z0, double dz0,
                    double zmax, const luna_solve_opts* opts, double* saves, double* steplog,
                    luna_solve_stats* stats);

/* Batched scan of independent instances in one persistent launch (replaces a sequential
 * Scans.runscan loop over prop_capillary calls, Scans.jl:275-494). All plans must share
 * one precision. Device buffers live in the batch; upload/run/download split the work so
 * the device-only part can be timed. */
int luna_b200_batch_create(luna_plan* const* plans, int n, const luna_solve_opts* opts, luna_batch** out);
int luna_b200_batch_upload(luna_batch* b, const double* const* linops, const double* const* y0,
                           const double* z0, const double* dz0, const double* zmax,
                           const double* const* zsave, const double* max_dt);
/* zsave (optional, NULL): per-instance [saveN] GridCondition points, e.g. range(0, zmax_i,
 * saveN) as Luna.run uses for each instance; max_dt (optional, NULL): per-instance step
 * limits (Luna.run's max_dz = zmax/2). NULL falls back to the batch-wide options. */
int luna_b200_batch_run(luna_batch* b, float* device_ms);
int luna_b200_batch_download(luna_batch* b, double* const* saves, double* const* y_out,
                             luna_solve_stats* stats);
int luna_b200_batch_steplog(luna_batch* b, int i, double* steplog);
/* Per-step statistics of instance i ([LUNA_NSTATS * stats_cap] doubles; stats.nstats rows
 * are valid) — the `stats` group a MemoryOutput collects through Stats.default. */
int luna_b200_batch_stats(luna_batch* b, int i, double* stats);
/* How a batch is scheduled (no counterpart in the reference): kernel launches per
 * luna_b200_batch_run, instances integrated on response clusters (mixed precision,
 * Raman buffers larger than one CTA's shared memory) and the number of clusters. */
int luna_b200_batch_info(luna_batch* b, int* kernels_per_run, int* cluster_instances, int* clusters);
/* Processing order of a batch (no counterpart in the reference): instances with a larger
 * priority[i] are started first ([n] doubles, e.g. an estimate of the instance's work). */
int luna_b200_batch_set_priority(luna_batch* b, const double* priority);
/* Scheduling record of the last run (no counterpart in the reference): per instance the
 * start and end of its integration in seconds from the earliest start ([2*n] doubles) and
 * the SM that integrated it ([n] ints, may be NULL). */
int luna_b200_batch_timeline(luna_batch* b, double* begin_end_s, int* sm);
/* Shape of every instance for the next luna_b200_batch_set_priority (no counterpart in the
 * reference; an autotuner's decision): [n] ints, 0 = decided from the work estimates (an
 * eligible instance whose estimate is at least the mean load of an SM runs on a cluster of
 * 8 CTAs, at least four times that on a cluster of 16 where the grid allows one),
 * 1 = one CTA, 2 = a cluster of 8 CTAs, 3 = a cluster of 16 CTAs, each when the instance is
 * eligible (the next smaller shape otherwise); NULL restores 0 for all. */
int luna_b200_batch_set_shapes(luna_batch* b, const int* shape);
/* Step sequence of instance i for the next runs (a verification aid, no counterpart in the
 * reference; the per-instance form of luna_solve_opts.replay): [2*nreplay] doubles, the
 * (dz, accepted) of each step as luna_b200_batch_steplog records them (columns 1 and 3);
 * nreplay = 0 removes it. Takes effect at the next luna_b200_batch_upload. */
int luna_b200_batch_set_replay(luna_batch* b, int i, const double* replay, long long nreplay);
void luna_b200_batch_destroy(luna_batch* b);

/* ---------------------------------------------------------------- radial transform
 * TransRadial (NonlinearRHS.jl:406-474) on a field-resolved or envelope grid with an order-0 QDHT of
 * Nr points (Hankel.jl QDHT(R, N, dim=2), as built by Luna.setup for radial symmetry,
 * Luna.jl:239-279). Fields are column-major Nw x Nr complex arrays (Julia's
 * Matrix{ComplexF64}): element (ω, k) at k*Nw + ω. */
typedef struct {
    int Nr;                /* radial points QDHT.N                                        */
    const double* Mi;      /* [Nr*Nr] row-major: E(r_n) = sum_m Mi[n*Nr+m] E(k_m)  (QDHT \ E) */
    const double* Mf;      /* [Nr*Nr] row-major: P(k_m) = sum_n Mf[m*Nr+n] P(r_n)  (QDHT * P) */
    const double* outfac;  /* [2*Nw*Nr] crop scale x ωwin (-iω) / (2 normfun(ω, k))        */
} luna_radial_desc;

typedef struct luna_radial_plan luna_radial_plan;

/* Replaces the TransRadial constructor (NonlinearRHS.jl:430-458). The grid descriptor is
 * that of one radial column (kind 0 or 1; its outfac is ignored, in_scale = pad scale / No);
 * responses as for luna_b200_plan_create, applied column by column as Et_to_Pt! does with
 * its CartesianIndices (NonlinearRHS.jl:137-141). */
int luna_b200_radial_plan_create(const luna_grid_desc* grid, const luna_resp_desc* resps, int nresp,
                                 const luna_radial_desc* radial, int precision, luna_radial_plan** out);
void luna_b200_radial_plan_destroy(luna_radial_plan* plan);
/* Attach (or, with grad == NULL, remove) a gas fill gradient: make_linop(grid, q, nfun)
 * (LinearOps.jl:174-226) and norm_radial (NonlinearRHS.jl:494-524) with
 * nfun(ω; z) = sqrt(1 + γ(ω) ρ(z)) and the densityfun(z) of TransRadial, ρ(z) the fill law
 * of luna_gradient_desc (npts, two_point, Z, P, P2, dens_a, dens_b). Fields used: gam [Nw]
 * γ(ω) on sidx, wc [Nw] ω/c on sidx (0 elsewhere), om [Nw] ω, ofs [2*Nw] crop scale x
 * ωwin (-iω)/2, fd_xc/fd_gam/fd_h12 for β1(z) (the 4-point central difference of
 * x/c n(x; z) at ω0, h = 1e-4 ω0), and on an envelope grid env_ref/ref_xc/ref_gam
 * (+ i β(ω0; z) without THG); kr2 [Nr] the QDHT's k_r^2, mu0w [Nw] μ0 ω. Then, at every
 * stage node, step end and save point:
 *   k2 = ((n ω/c))^2 on sidx (as n x (ω/c)), βsq = k2 - k_r^2,
 *   L = -i (sqrt(βsq) - β1 ω), or -i (-β1 ω) - min(sqrt|βsq|, 200) for βsq < 0,
 *   output factor = ρ(z) ofs / normfun, normfun = sqrt(βsq)/(μ0 ω) (1 where ω = 0 or βsq <= 0),
 * in IEEE-rounded operations in this order; the responses' coefficients are for ρ = 1 and
 * the linop argument of luna_b200_radial_solve is ignored (may be NULL). A Raman response
 * whose dephasing depends on the density is refused here. */
int luna_b200_radial_set_gradient(luna_radial_plan* plan, const luna_gradient_desc* grad, const double* kr2,
                                  const double* mu0w);
/* linop!(out, z) and the output factor of a radial plan with a gas fill gradient, evaluated
 * on the device as the solver does: host arrays of Nw*Nr complex (outfac may be NULL). */
int luna_b200_radial_linop(luna_radial_plan* plan, double z, double* linop, double* outfac);
/* (t::TransRadial)(nl, Eω, z) — NonlinearRHS.jl:466-474. Host arrays of Nw*Nr complex. */
int luna_b200_radial_rhs(luna_radial_plan* plan, double* nl, const double* Ew, double z);
int luna_b200_radial_rhs_device(luna_radial_plan* plan, double* nl_dev, const double* Ew_dev, double z,
                                void* stream);
/* The plan's QDHT along the radial index of an Nw x Nr complex device array (column-major):
 * forward != 0: Y = QDHT * X  (mul!(Y, QDHT, X), r -> k);  forward == 0: Y = QDHT \ X
 * (ldiv!, k -> r) — Hankel.jl's QDHT as called at NonlinearRHS.jl:468, 471. X and Y hold
 * complex FP64 for LUNA_PREC_FP64 plans and complex FP32 for LUNA_PREC_MIXED plans (where
 * the product runs as 3xBF16 tensor-core MMAs with FP32 accumulation); they must not
 * overlap and must be 8-byte aligned (LUNA_ERR_BAD_ARG otherwise). Enqueued on `stream`. */
int luna_b200_qdht_device(luna_radial_plan* plan, void* Y_dev, const void* X_dev, int forward, void* stream);
/* RK45.solve_precon driven by Luna.run (Luna.jl:358-391) for a radial problem: linop and
 * y_inout are Nw*Nr complex (LinearOps.make_const_linop(grid, q, nfun), LinearOps.jl:130-144),
 * saves [saveN*2*Nw*Nr] doubles, steplog as for luna_b200_solve. Host memory. */
int luna_b200_radial_solve(luna_radial_plan* plan, const double* linop, double* y_inout, double z0,
                           double dz0, double zmax, const luna_solve_opts* opts, double* saves,
                           double* steplog, luna_solve_stats* stats);

/* ---------------------------------------------------------------- modal transform
 * TransModal with full=false (NonlinearRHS.jl:148-302, built by Luna.setup for modes,
 * Luna.jl:173-199) on a field-resolved grid: nmodes capillary modes sharing the polar
 * limits (0, a), npol polarisation components (Modes.ToSpace, Modes.jl:411-442), the
 * radial integral of the projected polarisation by the p-adaptive Clenshaw-Curtis rule of
 * Cubature.pcubature_v (NonlinearRHS.jl:294-298) with the L2 error norm. Level l of the rule
 * has 2^(l+1)+1 points on [0, a]; the end points contribute nothing, the other points are
 * numbered in evaluation order ("slots": slot 0 the centre, then the 2^l points each level
 * l >= 1 adds), nslots = 2^nlevels - 1. Level l is accepted when the L2 norm of its
 * difference from level l-1 (level -1: the midpoint rule) is <= atol or <= rtol times its
 * own L2 norm, or when it is the last level (the evaluation limit mfcn). Fields are
 * column-major Nw x nmodes complex arrays (Julia's Matrix{ComplexF64}). */
#define LUNA_MODAL_MAX_MODES 16
#define LUNA_MODAL_MAX_LEVELS 9
typedef struct {
    int nmodes;            /* modes (columns of Eω), 1..LUNA_MODAL_MAX_MODES               */
    int npol;              /* 1 (components :x or :y) or 2 (:xy; Kerr response only)      */
    int nlevels;           /* cubature levels 0..nlevels-1, 1..LUNA_MODAL_MAX_LEVELS        */
    const double* ems;     /* [nslots*nmodes*npol] Exy(mode, (r_s, 0))[component] at slot s */
    const double* wts;     /* [nlevels*nslots] weight of slot s in level l's rule, 2πr_s and
                              the half-width a/2 included (0 for slots beyond level l)     */
    double wlow;           /* weight of slot 0 in the midpoint rule (level 0's comparison) */
    double rtol, atol;     /* pcubature reltol and abstol                                  */
    const double* outfac;  /* [2*Nw*nmodes] crop scale x ωwin x norm! per mode column     */
} luna_modal_desc;

typedef struct luna_modal_plan luna_modal_plan;

/* Replaces the TransModal constructor (NonlinearRHS.jl:203-216). The grid descriptor is
 * that of one point (kind 0 or 1; its outfac is ignored, in_scale = pad scale / No); responses
 * as for luna_b200_plan_create without the no-THG forms (and without plasma on an envelope
 * grid, as in the reference): with npol = 1 Kerr, plasma and
 * Raman (scalar RamanPolar on the modal field, Nonlinear.jl:284-290); with npol = 2 Kerr
 * (KerrVector!) and plasma (PlasmaVector!, Nonlinear.jl:144-162; vector Raman is not
 * implemented in the reference either). */
int luna_b200_modal_plan_create(const luna_grid_desc* grid, const luna_resp_desc* resps, int nresp,
                                const luna_modal_desc* modal, int precision, luna_modal_plan** out);
void luna_b200_modal_plan_destroy(luna_modal_plan* plan);
/* (t::TransModal)(nl, Eω, z) — NonlinearRHS.jl:284-302. Host arrays of Nw*nmodes complex;
 * nevals (may be NULL) receives the integrand evaluations the cubature took. */
int luna_b200_modal_rhs(luna_modal_plan* plan, double* nl, const double* Ew, double z, int* nevals);
int luna_b200_modal_rhs_device(luna_modal_plan* plan, double* nl_dev, const double* Ew_dev, double z,
                               void* stream);
/* RK45.solve_precon driven by Luna.run (Luna.jl:358-391) for a modal problem: linop and
 * y_inout are Nw*nmodes complex (LinearOps.make_const_linop(grid, modes, λ0),
 * LinearOps.jl:401-415), saves [saveN*2*Nw*nmodes] doubles, steplog as for luna_b200_solve. */
int luna_b200_modal_solve(luna_modal_plan* plan, const double* linop, double* y_inout, double z0,
                          double dz0, double zmax, const luna_solve_opts* opts, double* saves,
                          double* steplog, luna_solve_stats* stats);

/* Allocation-free variant of luna_b200_rhs_device. It has no counterpart in the reference:
 * it serves host programs that must not allocate device memory while they run (for
 * example a solver inside an allocator-managed runtime, or a process whose device memory
 * is owned by another framework's caching pool, where a cudaMalloc could fail or
 * fragment the pool). It allocates nothing: its scratch is a fixed buffer of
 * LUNA_NOALLOC_SCRATCH_BYTES in the library's static device memory, held by every device
 * that loads the library until the process exits. The plan (created beforehand) and the
 * caller's device buffers nl_dev/Ew_dev ([2*Nw] doubles) and status_dev (one int, may be
 * NULL; receives LUNA_OK or LUNA_FIELD_ABOVE_EMAX) are the only other memory it touches.
 * The first call on a device resolves the buffer's device address; make that first call
 * before any stream capture. Plans whose transforms need more scratch than the buffer are
 * rejected with LUNA_ERR_UNSUPPORTED. All calls share the one buffer: calls that overlap on
 * the GPU (different streams, or different host threads) race and must be serialised. */
#define LUNA_NOALLOC_SCRATCH_BYTES (1u << 20)
int luna_b200_rhs_device_noalloc(luna_plan* plan, double* nl_dev, const double* Ew_dev, double z,
                                 void* stream, int* status_dev);

const char* luna_b200_last_error(void);
int luna_b200_version(void);

#ifdef __cplusplus
}
#endif
#endif
