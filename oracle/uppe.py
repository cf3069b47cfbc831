"""FP64 numpy restatement of the UPPE hot path (test infrastructure only).

Every function cites the reference file:line it follows (Luna.jl v0.6.2). The
transform object it consumes is the same ``TransModeAvg`` description that the device
plan is built from, so both sides see identical inputs.
"""
import math

import numpy as np

# ------------------------------------------------------------------- Maths.cumtrapz!

def cumtrapz(y, dx):
    """Running trapezoid integral (Maths.jl:323-328).

    ``out[i] = out[i-1] + 1/2*(y[i-1]+y[i])*dx`` evaluated left to right; numpy's
    cumsum is a sequential left-to-right sum, so the rounding matches the reference.
    """
    inc = np.empty_like(y)
    inc[0] = 0.0
    inc[1:] = (0.5 * (y[:-1] + y[1:])) * dx
    return np.cumsum(inc)


# ------------------------------------------------------------------- rate functions

def ppt_rate(spl, E):
    """PPT log-rate spline closure (Ionisation.jl:257-270, Maths.jl:764-848).

    Raises ``ValueError`` for fields above the table maximum, as the reference errors.
    """
    aE = np.abs(E)
    out = np.zeros_like(aE)
    if np.any(aE > spl.Emax):
        raise ValueError(f"Field strength {aE.max()} V/m exceeds maximum for PPT "
                         f"ionisation rate ({spl.Emax} V/m).")
    m = aE >= spl.Emin
    x0 = aE[m]
    x, y, D = spl.x, spl.y, spl.D
    n = len(x)
    xmin, xmax = x[0], x[-1]
    # uniform-axis index function (Maths.jl:772-774), 1-based
    i1 = np.where(x0 <= xmin, 2,
                  np.where(x0 >= xmax, n,
                           np.ceil((x0 - xmin) / (xmax - xmin) * (n - 1)).astype(np.int64) + 1))
    i = i1 - 1  # 0-based index of the knot above x0
    xi, xim = x[i], x[i - 1]
    yi, yim = y[i], y[i - 1]
    Di, Dim = D[i], D[i - 1]
    t = (x0 - xim) / (xi - xim)
    val = (yim + Dim * t + (3 * (yi - yim) - 2 * Dim - Di) * t ** 2
           + (2 * (yim - yi) + Dim + Di) * t ** 3)
    val = np.where(x0 == xi, yi, np.where(x0 == xim, yim, val))
    out[m] = np.exp(val)
    return out


def adk_rate(r, E):
    """ADK closure (Ionisation.jl:43-59)."""
    aE = np.abs(E)
    out = np.zeros_like(aE)
    m = aE >= r.thr
    x = aE[m]
    out[m] = (r.w_p * r.cn_sq * (4 * r.w_p / (r.w_t_prefac * x)) ** (2 * r.nstar - 1)
              * np.exp(-4 / 3 * r.w_p / (r.w_t_prefac * x)))
    return out


def rate(ratefunc, E):
    if ratefunc.kind == "adk":
        return adk_rate(ratefunc, E)
    return ppt_rate(ratefunc, E)


# ------------------------------------------------------------------- responses

EPS0 = 8.854187817620389e-12
E_RATIO = 1.6021766208e-19 ** 2 / 9.10938356e-31


def kerr_field(out, E, rho, g3):
    """Nonlinear.jl:8-10, 24-34."""
    out += (rho * EPS0 * g3) * E ** 3


def kerr_env(out, E, rho, g3):
    """Nonlinear.jl:47-49, 63-73."""
    out += 3 / 4 * (rho * EPS0 * g3) * np.abs(E) ** 2 * E


def plasma(out, E, rho, p):
    """PlasmaCumtrapz scalar response (Nonlinear.jl:121-133, 164-177)."""
    r = rate(p.ratefunc, E)
    frac = cumtrapz(r, p.δt)
    frac = p.preionfrac + 1 - np.exp(-frac)
    phase = frac * E_RATIO * E
    J = cumtrapz(phase, p.δt)
    nz = np.abs(E) > 0
    J[nz] += p.ionpot * r[nz] * (1 - frac[nz]) / E[nz]
    P = cumtrapz(J, p.δt)
    out += rho * P


def hilbert(x):
    """Maths.hilbert (Maths.jl:560-569): analytic signal of a real array of even length n:
    FFT, bins 1..n/2-1 doubled, bins n/2..n-1 zeroed, inverse FFT."""
    xf = np.fft.fft(x)
    n1 = len(x) // 2
    xf[1:n1] *= 2
    xf[n1:] = 0
    return np.fft.ifft(xf)


def kerr_field_nothg(out, E, rho, g3):
    """Kerr_field_nothg (Nonlinear.jl:36-45): 3/4 ρ ε0 γ3 |hilbert(E)|² E."""
    out += rho * 3 / 4 * EPS0 * g3 * np.abs(hilbert(E)) ** 2 * E


def kerr_env_thg(out, E, rho, r):
    """Kerr_env_thg (Nonlinear.jl:75-84): ρ ε0 γ3/4 (3|E|² + exp(2iω0t) E²) E."""
    out += rho * EPS0 * r.γ3 / 4 * (3 * np.abs(E) ** 2 + r.C * E ** 2) * E


def raman_h(resp, rho):
    """CombinedRamanResponse(ht, rho) (Raman.jl:256-262)."""
    return resp.r.h(rho)


def raman_field(out, E, rho, resp):
    """RamanPolarField (Nonlinear.jl:282-333) on a 2x zero-padded grid; E² is
    1/2 |hilbert(E)|² without third-harmonic generation (sqr!, Nonlinear.jl:267-274)."""
    n = len(E)
    h = np.zeros(2 * n)
    h[:n] = raman_h(resp, rho)
    hw = np.fft.rfft(h)
    E2 = np.zeros(2 * n)
    E2[:n] = E ** 2 if getattr(resp, "thg", True) else 0.5 * np.abs(hilbert(E)) ** 2
    Pw = hw * np.fft.rfft(E2) * resp.dt
    P = np.fft.irfft(Pw, 2 * n)
    out += rho * E * P[:n]


def raman_env(out, E, rho, resp):
    """RamanPolarEnv (Nonlinear.jl:276-279, 282-333) with complex FFTs of length 2n."""
    n = len(E)
    h = np.zeros(2 * n, dtype=np.complex128)
    h[:n] = raman_h(resp, rho)
    hw = np.fft.fft(h)
    E2 = np.zeros(2 * n, dtype=np.complex128)
    E2[:n] = 0.5 * np.abs(E) ** 2
    Pw = hw * np.fft.fft(E2) * resp.dt
    P = np.fft.ifft(Pw)
    out += rho * E * P[:n]


def et_to_pt(Et, resp, rho):
    """Et_to_Pt! (NonlinearRHS.jl:121-126): zero, then accumulate each response in order."""
    Pt = np.zeros_like(Et)
    for r in resp:
        if r.kind == "kerr_field":
            kerr_field(Pt, Et, rho, r.γ3)
        elif r.kind == "kerr_env":
            kerr_env(Pt, Et, rho, r.γ3)
        elif r.kind == "kerr_field_nothg":
            kerr_field_nothg(Pt, Et, rho, r.γ3)
        elif r.kind == "kerr_env_thg":
            kerr_env_thg(Pt, Et, rho, r)
        elif r.kind == "plasma":
            plasma(Pt, Et, rho, r)
        elif r.kind == "raman_field":
            raman_field(Pt, Et, rho, r)
        elif r.kind == "raman_env":
            raman_env(Pt, Et, rho, r)
        else:
            raise ValueError(r.kind)
    return Pt


# ------------------------------------------------------------------- transform

def to_time(grid, Ew):
    """to_time! (NonlinearRHS.jl:16-32): zero-pad, rescale and inverse-transform."""
    Nw = len(Ew)
    if grid.kind == "real":
        Nwo = len(grid.ωo)
        scale = (Nwo - 1) / (Nw - 1)
        Ewo = np.zeros(Nwo, dtype=np.complex128)
        Ewo[:Nw] = scale * Ew
        return np.fft.irfft(Ewo, grid.No)
    No = grid.No
    scale = No / Nw
    h = Nw // 2
    Ewo = np.zeros(No, dtype=np.complex128)
    Ewo[:h] = scale * Ew[:h]
    Ewo[No - h:] = scale * Ew[Nw - h:]
    return np.fft.ifft(Ewo)


def to_freq(grid, Pt, Nw):
    """to_freq! (NonlinearRHS.jl:39-53): forward transform, crop and rescale."""
    if grid.kind == "real":
        Pwo = np.fft.rfft(Pt)
        scale = (Nw - 1) / (len(Pwo) - 1)
        return scale * Pwo[:Nw]
    No = len(Pt)
    Pwo = np.fft.fft(Pt)
    scale = Nw / No
    h = Nw // 2
    out = np.empty(Nw, dtype=np.complex128)
    out[:h] = scale * Pwo[:h]
    out[Nw - h:] = scale * Pwo[No - h:]
    return out


NLSCALE = math.sqrt(EPS0 * 299792458.0 / 2)


def trans_mode_avg(t, Ew, z):
    """(t::TransModeAvg)(nl, Eω, z) (NonlinearRHS.jl:362-373); with a pressure gradient the
    density is densityfun(z) and the normalisation uses βfun!(β, z) (:375-387)."""
    g = t.grid
    Et = to_time(g, Ew)
    Et = Et / (NLSCALE * math.sqrt(t.aeff))
    zdep = getattr(t, "kind", "") == "modeavg_z"
    if zdep:  # aeff(z) of a taper (Modes.Aeff(m; z))
        Et = to_time(g, Ew) / (NLSCALE * math.sqrt(t.aefffun(z)))
    Pt = et_to_pt(Et, t.resp, t.densityfun(z) if zdep else t.density)
    Pt = Pt * g.towin
    nl = to_freq(g, Pt, len(Ew))
    s = g.sidx
    if zdep:
        nl[s] = nl[s] * t.norm_factor(z)[s]
        return nl
    nl[s] = nl[s] * (t.norm.pre[s] * math.sqrt(t.aeff))
    nl[s] = nl[s] * g.ωwin[s]
    return nl


def trans_radial(t, Ew, z):
    """(t::TransRadial)(nl, Eω, z) (NonlinearRHS.jl:466-474) for a field-resolved or an
    envelope grid: Ew is (Nω, Nr) in (ω, k) space; the responses act on each radial column
    (Et_to_Pt! with CartesianIndices, NonlinearRHS.jl:137-141)."""
    g, q = t.grid, t.q
    Nw, Nr = Ew.shape
    zdep = getattr(t, "kind", "") == "radial_z"   # densityfun(z), normfun(z) of a gas fill gradient
    rho = t.densityfun(z) if zdep else t.density
    Et = np.stack([to_time(g, Ew[:, i]) for i in range(Nr)], axis=1)  # to_time! along dim 1
    Er = q.inverse(Et, axis=1)                     # ldiv!(Eto, QDHT, Eto): k -> r
    Pr = np.zeros_like(Er)
    for i in range(Nr):                            # Et_to_Pt! per radial column
        Pr[:, i] = et_to_pt(Er[:, i], t.resp, rho)
    Pr = Pr * g.towin[:, None]
    Pk = q.forward(Pr, axis=1)                     # mul!(Pto, QDHT, Pto): r -> k
    nl = np.stack([to_freq(g, Pk[:, i], Nw) for i in range(Nr)], axis=1)  # to_freq!
    return nl * (t.output_factor_z(z) if zdep else t.output_factor())


def kerr_vector(out, E, rho, g3):
    """KerrVector! (Nonlinear.jl:12-21): E is (n, 2)."""
    fac = rho * EPS0 * g3
    s = E[:, 0] ** 2 + E[:, 1] ** 2
    out[:, 0] += fac * s * E[:, 0]
    out[:, 1] += fac * s * E[:, 1]


def plasma_vector(out, E, rho, p):
    """PlasmaVector! (Nonlinear.jl:144-162): the rate and ionisation fraction from |E| of
    the (n, 2) field, the phase, current and polarisation per component."""
    Em = np.hypot(E[:, 0], E[:, 1])
    r = rate(p.ratefunc, Em)
    frac = cumtrapz(r, p.δt)
    frac = p.preionfrac + 1 - np.exp(-frac)
    for c in range(2):
        phase = frac * E_RATIO * E[:, c]
        J = cumtrapz(phase, p.δt)
        nz = np.abs(Em) > 0
        J[nz] += p.ionpot * r[nz] * (1 - frac[nz]) / Em[nz] ** 2 * E[nz, c]
        out[:, c] += rho * cumtrapz(J, p.δt)


def et_to_pt_modal(Er, resp, rho):
    """Et_to_Pt! on the (n, npol) real-space field of one point: scalar responses for one
    component (Nonlinear.jl:24-34, 164-177 with size(Et, 2) == 1), vector Kerr and vector
    plasma for two."""
    if Er.shape[1] == 1:
        return et_to_pt(Er[:, 0], resp, rho)[:, None]
    Pr = np.zeros_like(Er)
    for r in resp:
        if r.kind == "kerr_field":
            kerr_vector(Pr, Er, rho, r.γ3)
        elif r.kind == "kerr_env":
            kerr_vector_env(Pr, Er, rho, r.γ3)
        elif r.kind == "plasma":
            plasma_vector(Pr, Er, rho, r)
        else:
            raise NotImplementedError(r.kind)
    return Pr


def kerr_vector_env(out, E, rho, g3):
    """KerrVectorEnv! (Nonlinear.jl:52-63): E is the (n, 2) complex envelope."""
    fac = rho * EPS0 * g3
    Ex, Ey = E[:, 0], E[:, 1]
    Ex2, Ey2 = np.abs(Ex) ** 2, np.abs(Ey) ** 2
    out[:, 0] += 3 / 4 * fac * ((Ex2 + 2 / 3 * Ey2) * Ex + 1 / 3 * np.conj(Ex) * Ey ** 2)
    out[:, 1] += 3 / 4 * fac * ((Ey2 + 2 / 3 * Ex2) * Ey + 1 / 3 * np.conj(Ey) * Ex ** 2)


def clenshaw_curtis_moments(n):
    """Weights of the (n+1)-point Clenshaw-Curtis rule on [-1, 1] (nodes cos(jπ/n)) from its
    definition: the rule integrates the Chebyshev polynomials T_0..T_n exactly,
    sum_j w_j cos(kjπ/n) = ∫ T_k = (1 + (-1)^k)/(1 - k²) (0 for k = 1)."""
    j = np.arange(n + 1)
    A = np.cos(np.outer(j, j) * math.pi / n)  # A[k, j] = T_k(x_j)
    k = j.astype(np.float64)
    with np.errstate(divide="ignore"):
        mom = np.where(k % 2 == 0, 2.0 / (1.0 - k * k), 0.0)
    return np.cos(j * math.pi / n), np.linalg.solve(A, mom)


def pcubature(f, lo, hi, rtol, atol, maxevals):
    """One-dimensional ``Cubature.pcubature_v(fdim, f, (lo,), (hi,); reltol, abstol, maxevals,
    error_norm=Cubature.L2)`` as called at NonlinearRHS.jl:294-298. Cubature.jl (compat 1.5.1,
    Project.toml:62; not vendored, so the exact version is unpinned) wraps S. G. Johnson's cubature library; its p-adaptive routine,
    as published, doubles the degree of nested Clenshaw-Curtis rules until the error estimate
    (the difference from the previous rule) meets the tolerance. Restated here: level m uses
    the 2^(m+1)+1-point rule, level -1 the midpoint rule; the error of level m is
    ||I_m - I_{m-1}||_2 over the fdim components; converged when it is <= abstol or
    <= reltol ||I_m||_2; the next level is only evaluated while its points fit in
    maxevals. Integrand values are cached per point. Returns (I_m, error, evaluations)."""
    c, h = (lo + hi) / 2, (hi - lo) / 2
    cache = {}
    DEPTH = 1 << 12

    def F(j, n):  # node cos(jπ/n), keyed on the finest grid
        key = j * (DEPTH // n)
        if key not in cache:
            cache[key] = f(c + h * math.cos(j * math.pi / n))
        return cache[key]

    Ilow = h * 2.0 * F(1, 2)
    m = 0
    while True:
        n = 2 << m
        _, w = clenshaw_curtis_moments(n)
        I = h * sum(w[j] * F(j, n) for j in range(n + 1))
        err = float(np.linalg.norm(I - Ilow))
        if err <= atol or err <= rtol * float(np.linalg.norm(I)):
            break
        if (2 << (m + 1)) + 1 > maxevals or (2 << (m + 1)) > DEPTH:
            break
        Ilow = I
        m += 1
    return I, err, len(cache)


# Genz-Malik degree-7 rule with its embedded degree-5 rule in two dimensions (A. C. Genz and
# A. A. Malik, J. Comput. Appl. Math. 6, 295 (1980)); weights for a region of volume V sum
# to one: I = V * sum(w f).
_GM_L2, _GM_L3, _GM_L4, _GM_L5 = math.sqrt(9 / 70), math.sqrt(9 / 10), math.sqrt(9 / 10), math.sqrt(9 / 19)
_GM_W7 = ((12824 - 9120 * 2 + 400 * 4) / 19683, 980 / 6561, (1820 - 400 * 2) / 19683, 200 / 19683,
          6859 / 19683 / 4)
_GM_W5 = ((729 - 950 * 2 + 50 * 4) / 729, 245 / 486, (265 - 100 * 2) / 1458, 25 / 729)


def _gm_region(f, c, h):
    """Integral, error vector and split dimension of the box c ± h (2-D Genz-Malik)."""
    f0 = f(c[0], c[1])
    s2, s3, d2, d3 = [], [], [], []
    for i in range(2):
        e = [0.0, 0.0]
        e[i] = 1.0
        a2 = [f(c[0] + s * _GM_L2 * h[0] * e[0], c[1] + s * _GM_L2 * h[1] * e[1]) for s in (1, -1)]
        a3 = [f(c[0] + s * _GM_L3 * h[0] * e[0], c[1] + s * _GM_L3 * h[1] * e[1]) for s in (1, -1)]
        s2.append(a2[0] + a2[1])
        s3.append(a3[0] + a3[1])
        # fourth difference along dimension i: the split criterion
        d = (a2[0] + a2[1] - 2 * f0) - (_GM_L2 / _GM_L3) ** 2 * (a3[0] + a3[1] - 2 * f0)
        d2.append(float(np.linalg.norm(d)))
    s4 = sum(f(c[0] + sx * _GM_L4 * h[0], c[1] + sy * _GM_L4 * h[1]) for sx in (1, -1) for sy in (1, -1))
    s5 = sum(f(c[0] + sx * _GM_L5 * h[0], c[1] + sy * _GM_L5 * h[1]) for sx in (1, -1) for sy in (1, -1))
    V = 4 * h[0] * h[1]
    S2, S3 = s2[0] + s2[1], s3[0] + s3[1]
    I7 = V * (_GM_W7[0] * f0 + _GM_W7[1] * S2 + _GM_W7[2] * S3 + _GM_W7[3] * s4 + _GM_W7[4] * s5)
    I5 = V * (_GM_W5[0] * f0 + _GM_W5[1] * S2 + _GM_W5[2] * S3 + _GM_W5[3] * s4)
    split = 0 if d2[0] >= d2[1] else 1
    return I7, np.abs(I7 - I5), split


def hcubature2(f, lo, hi, rtol, atol, maxevals):
    """Two-dimensional ``Cubature.hcubature_v(fdim, f, lo, hi; reltol, abstol, maxevals,
    error_norm=Cubature.L2)`` as called at NonlinearRHS.jl:287-293 (full=true). Restated from
    the published h-adaptive algorithm of the cubature library (Cubature.jl compat 1.5.1,
    not vendored, unpinned): the regions form a heap on their error norm; while the summed
    error vector's L2 norm exceeds max(abstol, reltol ||I||) and evaluations remain, the
    regions with the largest errors are taken until the rest would meet the tolerance, each
    is bisected along the dimension of largest fourth difference and both halves are
    evaluated with the 17-point rule. Returns (I, error vector, evaluations)."""
    import heapq
    c = [(lo[0] + hi[0]) / 2, (lo[1] + hi[1]) / 2]
    h = [(hi[0] - lo[0]) / 2, (hi[1] - lo[1]) / 2]
    I, E, sp = _gm_region(f, c, h)
    heap = [(-float(np.linalg.norm(E)), 0, c, h, I, E, sp)]
    nev, uid = 17, 1
    tot_I, tot_E = I.copy(), E.copy()

    def ok(err, val):
        n = float(np.linalg.norm(err))
        return n <= atol or n <= rtol * float(np.linalg.norm(val))

    while not ok(tot_E, tot_I) and (not maxevals or nev < maxevals):
        take, rest_E = [], tot_E.copy()
        while heap:
            item = heapq.heappop(heap)
            take.append(item)
            rest_E = rest_E - item[5]
            if ok(rest_E, tot_I):
                break
        for _, _, rc, rh, rI, rE, rsp in take:
            hh = list(rh)
            hh[rsp] /= 2
            for s in (-1, 1):
                cc = list(rc)
                cc[rsp] += s * hh[rsp]
                I2, E2, sp2 = _gm_region(f, cc, hh)
                nev += 17
                heapq.heappush(heap, (-float(np.linalg.norm(E2)), uid, cc, hh, I2, E2, sp2))
                uid += 1
        # totals summed afresh over the regions (in creation order), not updated in place
        regs = sorted(heap, key=lambda q: q[1])
        tot_I = sum(q[4] for q in regs)
        tot_E = sum(q[5] for q in regs)
    return tot_I, tot_E, nev


def trans_modal(t, Ew, z):
    """(t::TransModal)(nl, Eω, z) (NonlinearRHS.jl:234-302) for a field-resolved or envelope grid: Ew is
    (Nω, nmodes). Per point: to_space! (Modes.jl:458-495), to_time!, Et_to_Pt!, towin,
    to_freq!, ωwin, norm!, projection onto the modes (Prω Emsᵀ) and the weight (2πr at
    θ = 0 for full=false, r over (r, θ) for full=true); points on or outside (0, a) give
    zero."""
    g, ts = t.grid, t.ts
    Nw = Ew.shape[0]
    lo, hi = 0.0, t.a
    of = g.ωwin * t.norm

    def point(r, θ=0.0):
        if r <= lo or r >= hi:
            return np.zeros_like(Ew)
        Ems = ts.ems(r, θ)                               # (nmodes, npol)
        Erω = Ew @ Ems                                   # (Nω, npol)
        # to_time! / to_freq! per component (real: irfft/rfft; envelope: copy_scale_both!)
        Er = np.stack([to_time(g, Erω[:, k]) for k in range(Erω.shape[1])], axis=1)
        Pr = et_to_pt_modal(Er, t.resp, t.density) * g.towin[:, None]
        Prω = np.stack([to_freq(g, Pr[:, k], Nw) for k in range(Pr.shape[1])], axis=1)
        Prω = Prω * of[:, None]
        return 2 * math.pi * r * (Prω @ Ems.T)           # (Nω, nmodes)

    if getattr(t, "full", False):
        def point2(r, θ):
            if r <= lo or r >= hi:
                return np.zeros_like(Ew)
            return point(r, θ) / (2 * math.pi)    # weight r (polar), not 2πr
        val, err, nev = hcubature2(point2, (lo, 0.0), (hi, 2 * math.pi), t.rtol, t.atol, t.mfcn)
    else:
        val, err, nev = pcubature(point, lo, hi, t.rtol, t.atol, t.mfcn)
    t.oracle_nevals = nev
    return val


def rhs(t, Ew, z):
    kind = getattr(t, "kind", "")
    if kind in ("radial", "radial_z"):
        return trans_radial(t, Ew, z)
    if kind == "modal":
        return trans_modal(t, Ew, z)
    return trans_mode_avg(t, Ew, z)


# ------------------------------------------------------------------- RK45 (dopri)

# Butcher tableau, nodes, weights and dense-output coefficients (dopri.jl:2-28)
B = [[1 / 5],
     [3 / 40, 9 / 40],
     [44 / 45, -56 / 15, 32 / 9],
     [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
     [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
     [35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84]]
NODES = [1 / 5, 3 / 10, 4 / 5, 8 / 9, 1, 1]
B5 = [5179 / 57600, 0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40]
B4 = [35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0]
ERREST = [a - b for a, b in zip(B5, B4)]
INTERPC = np.array([
    [1, 0, 0, 0, 0, 0, 0],
    [-183 / 64, 0, 1500 / 371, -125 / 32, 9477 / 3392, -11 / 7, 3 / 2],
    [37 / 12, 0, -1000 / 159, 125 / 12, -729 / 106, 11 / 3, -4],
    [-145 / 128, 0, 1000 / 371, -375 / 64, 25515 / 6784, -55 / 28, 5 / 2]])


def weaknorm(yerr, y, yn, rtol, atol):
    """RK45.jl:343-354."""
    sy = np.sum(np.abs(y) ** 2)
    syn = np.sum(np.abs(yn) ** 2)
    syerr = np.sum(np.abs(yerr) ** 2)
    errwt = max(max(math.sqrt(sy), math.sqrt(syn)), atol)
    return math.sqrt(syerr) / rtol / errwt


class PreconStepper:
    """Interaction-picture embedded RK (RK45.jl:128-226, 249-297, 374-406)."""

    def __init__(self, f, linop, y0, t, dt, rtol=1e-6, atol=1e-10, safety=0.9,
                 max_dt=math.inf, min_dt=0.0, locextrap=True):
        self.f = f
        self.linop = linop
        y0 = np.array(y0, dtype=np.complex128)
        self.y = y0.copy()
        self.yn = y0.copy()
        self.ks = [None] * 7
        self.t = float(t)
        self.tn = float(t)
        self.dt = float(dt)
        self.dtn = float(dt)
        self.rtol, self.atol, self.safety = rtol, atol, safety
        self.max_dt, self.min_dt = max_dt, min_dt
        self.locextrap = locextrap
        self.ok = False
        self.err = 0.0
        self.errlast = 0.0
        self.nrhs = 0
        self.ks[0] = self.fbar(y0, self.t, self.t)

    def prop(self, y, t1, t2, bwd=False):
        """make_prop! (RK45.jl:271-297): a constant linop, or linop(z) evaluated at the later
        point t2 (re-evaluated only when t2 changes)."""
        d = (t1 - t2) if bwd else (t2 - t1)
        if callable(self.linop):
            if getattr(self, "_lastt2", None) != t2:
                self._lin = self.linop(t2)
                self._lastt2 = t2
            return y * np.exp(self._lin * d)
        return y * np.exp(self.linop * d)

    def fbar(self, ybar, t1, t2):
        """make_fbar! (RK45.jl:299-310)."""
        y = self.prop(ybar, t1, t2)
        out = self.f(y, t2)
        self.nrhs += 1
        return self.prop(out, t1, t2, True)

    def evaluate(self):
        """evaluate!(::PreconStepper) (RK45.jl:209-223)."""
        self.y = self.yn.copy()
        self.ks[0] = self.prop(self.ks[0], self.t, self.tn)
        self.dt = self.dtn
        self.t = self.tn
        for ii in range(6):
            yn = self.y.copy()
            for jj in range(ii + 1):
                if B[ii][jj] != 0:
                    yn = yn + (self.dt * B[ii][jj]) * self.ks[jj]
            self.ks[ii + 1] = self.fbar(yn, self.t, self.t + NODES[ii] * self.dt)

    def step(self):
        """step! (RK45.jl:167-192)."""
        self.evaluate()
        if self.locextrap:
            yn = self.y.copy()
            for jj in range(7):
                if B5[jj] != 0:
                    yn = yn + (self.dt * B5[jj]) * self.ks[jj]
            self.yn = yn
        yerr = np.zeros_like(self.y)
        for ii in range(7):
            if ERREST[ii] != 0:
                yerr = yerr + self.dt * self.ks[ii] * ERREST[ii]
        self.err = weaknorm(yerr, self.y, self.yn, self.rtol, self.atol)
        self.ok = self.err <= 1
        self.stepcontrol()
        if self.ok:
            self.tn = self.t + self.dt
            self.ks[0] = self.ks[6].copy()
        else:
            self.yn = self.y.copy()
        self.yn = self.prop(self.yn, self.t, self.tn)
        return self.ok

    def stepcontrol(self):
        """stepcontrolPI! + steplims! (RK45.jl:374-406)."""
        b1 = 3 / 5 / 5
        b2 = -1 / 5 / 5
        eps = 0.8
        if self.ok:
            if self.errlast == 0:
                self.errlast = self.err
            if self.err == 0:
                fac = 1.5
            else:
                fac = self.safety * (eps / self.err) ** b1 * (eps / self.errlast) ** b2
            self.dtn = fac * self.dt
            self.errlast = self.err
        else:
            if not math.isfinite(self.err):
                self.dtn = self.dt / 2
            else:
                self.dtn = self.dt * max(0.1, self.safety * self.err ** (-1 / 5))
        if self.dtn > self.max_dt:
            self.dtn = self.max_dt
        elif self.dtn < self.min_dt:
            self.dtn = self.min_dt
            self.ok = True

    def interpolate(self, ti):
        """Dense output (RK45.jl:249-268); ks[0] already holds k7 after an accepted step."""
        if ti > self.tn:
            raise ValueError("Attempting to extrapolate!")
        if ti == self.t:
            return self.y.copy()
        if ti == self.tn:
            return self.yn.copy()
        s = (ti - self.t) / self.dt
        sp = np.array([s, s * s, s * s * s, (s * s) * (s * s)])
        b = np.sum(sp[:, None] * INTERPC, axis=0)
        yi = np.zeros_like(self.y)
        for ii in range(7):
            yi = yi + self.ks[ii] * b[ii]
        out = self.y + self.dt * yi
        return self.prop(out, self.t, ti)


# ------------------------------------------------------------------- per-step statistics

STATS_KEYS = ("z", "dz", "ω0", "energy", "peakpower", "peakintensity", "fwhm_t_min",
              "fwhm_t_max", "electrondensity", "peak_ionisation_rate")


def _linterpx(x1, x2, y1, y2, val):
    """Maths.linterpx (Maths.jl:230-236)."""
    slope = (y2 - y1) / (x2 - x1)
    icpt = y1 - slope * x1
    return (val - icpt) / slope


def fwhm_linear(x, y, minmax):
    """Maths.fwhm / level_xings with method=:linear, baseline=false, level=0.5
    (Maths.jl:128-190); NaN where a crossing is missing."""
    val = 0.5 * np.max(y)
    maxidx = int(np.argmax(y))
    xmax = x[maxidx]
    n = len(y)
    try:
        if minmax == "min":
            li = np.nonzero((x < xmax) & (y < val))[0]
            ri = np.nonzero((x > xmax) & (y < val))[0]
            lefti, righti = int(li[-1]), int(ri[0])
            left = _linterpx(x[lefti], x[lefti + 1], y[lefti], y[lefti + 1], val)
            right = _linterpx(x[righti - 1], x[righti], y[righti - 1], y[righti], val)
        else:
            li = np.nonzero((x < xmax) & (y > val))[0]
            ri = np.nonzero((x > xmax) & (y > val))[0]
            lefti, righti = int(li[0]), int(ri[-1])
            if lefti - 1 < 0 or righti + 1 > n - 1:
                raise IndexError
            left = _linterpx(x[lefti - 1], x[lefti], y[lefti - 1], y[lefti], val)
            right = _linterpx(x[righti], x[righti + 1], y[righti], y[righti + 1], val)
        return abs(right - left)
    except IndexError:
        return math.nan


def _simpson_even(x, y):
    """NumericalIntegration.jl integrate(x, y, SimpsonEven()) for uniform x."""
    h = x[1] - x[0]
    r = (17 * (y[0] + y[-1]) + 59 * (y[1] + y[-2]) + 43 * (y[2] + y[-3]) + 49 * (y[3] + y[-4])) / 48
    return h * (r + np.sum(y[4:len(y) - 4]))


def stats_default(t, Ew, z, dz):
    """Stats.default for a mode-averaged field-resolved transform (Stats.jl:495-532): the
    spectral centroid ω0 (:18-24), energy from energyfuncs' energy_ω (Fields.jl:510-520),
    peak power and peak intensity of the analytic field (:86-100, :150-154, plan_analytic
    :434-462), FWHM min/max (:182-200) and, with a plasma response, the electron density and
    peak ionisation rate (:228-257)."""
    g = t.grid
    a2 = np.abs(Ew) ** 2
    w = g.ω
    out = {"z": z, "dz": dz}
    out["ω0"] = np.sum(w * a2) / np.sum(a2)
    out["energy"] = 2 * math.pi / (w[-1] ** 2) * _simpson_even(w, a2)
    N = g.N
    Ewa = np.zeros(N, dtype=np.complex128)
    n = len(Ew) - 1
    Ewa[:n] = 2 * Ew[:n]
    Eta = np.fft.ifft(Ewa)
    Pt = np.abs(Eta) ** 2
    zdep = getattr(t, "kind", "") == "modeavg_z"
    aeff = t.aefffun(z) if zdep else t.aeff
    out["peakpower"] = np.max(Pt)
    out["peakintensity"] = np.max(Pt) / aeff
    out["fwhm_t_min"] = fwhm_linear(g.t, Pt, "min")
    out["fwhm_t_max"] = fwhm_linear(g.t, Pt, "max")
    out["electrondensity"] = math.nan
    out["peak_ionisation_rate"] = math.nan
    for r in t.resp:
        if getattr(r, "kind", "") == "plasma":
            Eto = np.real(Eta) / math.sqrt(EPS0 * 299792458.0 * aeff / 2)
            rr = rate(r.ratefunc, Eto)
            frac = cumtrapz(rr, g.t[1] - g.t[0])
            rho = t.densityfun(z) if zdep else t.density
            out["electrondensity"] = (1 - math.exp(-frac[-1])) * rho
            out["peak_ionisation_rate"] = np.max(rr)
    return out


class RunResult:
    def __init__(self):
        self.z = []
        self.Eω = []
        self.stats = []  # Stats.default rows (STATS_KEYS) of every accepted step
        self.steps = 0
        self.accepted = []  # (t, dt, err) of every accepted step
        self.steps_all = []  # (dt, ok) of every step, accepted or not
        self.rejected = 0
        self.nrhs = 0


def run(t, grid, linop, Eω0, z0=0.0, init_dz=1e-4, max_dz=None, min_dz=0.0, rtol=1e-6,
        atol=1e-10, safety=0.9, saveN=201, repeat_limit=10, max_steps=None, stats=False):
    """Luna.run (Luna.jl:358-391) with a MemoryOutput on a GridCondition (Output.jl:65-82,
    490-502) and RK45.solve's loop (RK45.jl:27-89)."""
    max_dz = grid.zmax / 2 if max_dz is None else max_dz
    zgrid = np.linspace(z0, grid.zmax, saveN)
    res = RunResult()
    f = lambda y, z: rhs(t, y, z)
    s = PreconStepper(f, linop, Eω0, z0, init_dz, rtol=rtol, atol=atol, safety=safety,
                      max_dt=max_dz, min_dt=min_dz)
    saved = 0
    repeated = 0
    kind = grid.kind

    def stepfun(yn, z, dz):
        # Luna.jl:366-372: window in frequency, back to time, window in time, forward
        nonlocal saved
        ww = grid.ωwin if yn.ndim == 1 else grid.ωwin[:, None]
        tw = grid.twin if yn.ndim == 1 else grid.twin[:, None]
        y = yn * ww
        if kind == "real":
            Et = np.fft.irfft(y, grid.N, axis=0) * tw
            y = np.fft.rfft(Et, axis=0)
        else:
            Et = np.fft.ifft(y, axis=0) * tw
            y = np.fft.fft(Et, axis=0)
        s.yn = y
        if stats:  # MemoryOutput calls statsfun before the saves (Output.jl:65-82)
            d = stats_default(t, y, z, dz)
            res.stats.append([d[k] for k in STATS_KEYS])
        while saved < saveN and zgrid[saved] <= z:
            res.z.append(zgrid[saved])
            res.Eω.append(s.interpolate(zgrid[saved]))
            saved += 1

    # the output is initialised with the first save point at z0 when it is reached by
    # the first accepted step's condition check (z0 <= tn)
    while s.tn <= grid.zmax:
        ok = s.step()
        res.steps += 1
        res.steps_all.append((s.dt, 1.0 if ok else 0.0))
        if ok:
            res.accepted.append((s.t, s.dt, s.err))
            stepfun(s.yn, s.tn, s.dtn)
            repeated = 0
        else:
            res.rejected += 1
            repeated += 1
            if repeated > repeat_limit:
                raise RuntimeError(f"Reached limit for step repetition ({repeat_limit})")
        if max_steps is not None and res.steps >= max_steps:
            break
    res.nrhs = s.nrhs
    res.stats = np.array(res.stats)
    res.Eω = np.array(res.Eω)
    res.z = np.array(res.z)
    return res
