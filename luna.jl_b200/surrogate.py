"""Learned surrogate of the capillary scan family (the reference has no counterpart: it
always integrates).

An ensemble of multilayer perceptrons maps (energy, pressure, core radius, τfwhm, z, gas)
to the log10 spectral intensity on 512 log-spaced wavelength bins (150 nm - 4 µm, the
λ-Jacobian of ``Processing.getIω``, Processing.jl:544-557) and the temporal envelope
|E(t)|^2 of the analytic field on 256 samples over ±150 fs. It is trained on data the
batched solver generates and evaluated with the project's own kernels
(``luna.jl_b200/csrc/surrogate.cu``, declarations in ``include/luna_surrogate.h``):

* input: 8 standardised features (energy, pressure, radius, τfwhm, z, and gas as three
  indicator columns with He as the reference), Fourier features (the raw 8 plus sin and cos
  of 124 fixed random projections, 256 inputs);
* 6 linear layers, width 512, SiLU, 768 outputs (512 spectral + 256 envelope); BF16
  operands on the tensor cores, FP32 master weights and Adam;
* 4 members (different initialisation and data order); a query whose ensemble spread on
  the spectral outputs exceeds ``spread_limit`` decades goes back to the solver
  (``Surrogate.query``), as does a random audit fraction.

Spectra are normalised by the peak of the same run's input spectrum and floored at 1e-6
(6 decades), envelopes by the input peak power.
"""
import ctypes
import math
import os

import numpy as np

from . import physdata as pd

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libluna_surrogate.so")

NSPEC, NENV = 512, 256
NOUT = NSPEC + NENV
NFEAT = 8
NFOURIER = 124
NIN = 8 + 2 * NFOURIER  # 256
WIDTHS = (NIN, 512, 512, 512, 512, 512, NOUT)
LAMBDA = (150e-9, 4e-6)
TWIN = 150e-15
FLOOR = -6.0
GASES = ("He", "Ne", "Ar", "H2")

_lib = None


def load():
    """The kernel library; fails loudly when it is missing (there is no CPU path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with luna.jl_b200/build.py")
    lib = ctypes.CDLL(LIB_PATH)
    vp, i, ll, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_float, ctypes.c_double
    lib.luna_sg_linear_fwd.argtypes = [vp, ll, vp, vp, i, i, i, i, vp, vp, vp, i, vp, vp]
    lib.luna_sg_linear_bwd_data.argtypes = [vp, vp, vp, i, i, i, vp, i, vp, vp]
    lib.luna_sg_linear_bwd_weight.argtypes = [vp, vp, ll, i, i, i, vp, vp, i, vp, vp]
    lib.luna_sg_features.argtypes = [vp, i, vp, i, vp, i, vp]
    lib.luna_sg_mse.argtypes = [vp, vp, ll, i, i, vp, vp, i, vp]
    lib.luna_sg_adam.argtypes = [vp, vp, vp, vp, ll, f, f, f, f, i, vp, vp]
    lib.luna_sg_ensemble.argtypes = [vp, i, i, i, i, vp, vp, vp]
    _lib = lib
    return lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"{what} returned {rc}")


# ----------------------------------------------------------------------------- features
def raw_features(energy, pressure, radius, tau, z, gas):
    """Unstandardised inputs [n, 8] (gas as three indicators, He the reference)."""
    n = len(energy)
    x = np.zeros((n, NFEAT))
    x[:, 0] = np.asarray(energy) * 1e6
    x[:, 1] = pressure
    x[:, 2] = np.asarray(radius) * 1e6
    x[:, 3] = np.asarray(tau) * 1e15
    x[:, 4] = z
    g = np.asarray(gas)
    for j, name in enumerate(GASES[1:]):
        x[:, 5 + j] = (g == name)
    return x


class Targets:
    """Spectral and envelope targets of the saved fields of one frequency grid: a matrix
    averaging |Eω|^2 ω^2/(2πc) over each of the 512 log-spaced λ bins, and the analytic
    field's power interpolated onto 256 times (torch on the GPU)."""

    def __init__(self, grid, device="cuda"):
        import torch
        self.torch = torch
        ω = np.asarray(grid.ω)
        # 512 log-spaced wavelength bins; each target is the mean of the λ-Jacobian-weighted
        # intensity over the grid frequencies inside its bin (linear interpolation at the
        # bin centre where a bin holds no grid frequency), i.e. the spectrum downsampled
        # rather than sampled, so fringes finer than a bin do not alias
        edges = np.geomspace(LAMBDA[0], LAMBDA[1], NSPEC + 1)
        lam = np.sqrt(edges[:-1] * edges[1:])
        wq = 2 * np.pi * pd.c / lam
        j = np.clip(np.searchsorted(ω, wq) - 1, 0, len(ω) - 2)
        f = (wq - ω[j]) / (ω[j + 1] - ω[j])
        M = np.zeros((NSPEC, len(ω)))
        whi = 2 * np.pi * pd.c / edges[:-1]
        wlo = 2 * np.pi * pd.c / edges[1:]
        for b in range(NSPEC):
            inside = np.nonzero((ω >= wlo[b]) & (ω < whi[b]))[0]
            if len(inside):
                M[b, inside] = 1.0 / len(inside)
            else:
                M[b, j[b]] = 1 - f[b]
                M[b, j[b] + 1] = f[b]
        jac = ω ** 2 / (2 * np.pi * pd.c)
        self.M = torch.tensor(M * jac[None, :], dtype=torch.float64, device=device)
        self.N = grid.N
        t = np.asarray(grid.t)
        tq = np.linspace(-TWIN, TWIN, NENV)
        k = np.clip(np.searchsorted(t, tq) - 1, 0, len(t) - 2)
        g = (tq - t[k]) / (t[k + 1] - t[k])
        T = np.zeros((NENV, len(t)))
        T[np.arange(NENV), k] = 1 - g
        T[np.arange(NENV), k + 1] = g
        self.T = torch.tensor(T, dtype=torch.float64, device=device)

    def __call__(self, saves, ref_spec=None, ref_env=None):
        """saves: complex128 tensor [nz, Nw]; returns (log10 spectrum [nz, 512], envelope
        [nz, 256]) normalised by the first save's peaks (or the ones given)."""
        torch = self.torch
        Iw = saves.real ** 2 + saves.imag ** 2
        Il = Iw @ self.M.T
        # analytic signal on the coarse grid: twice the positive frequencies, time centred
        a = torch.zeros((saves.shape[0], self.N), dtype=torch.complex128, device=saves.device)
        a[:, : saves.shape[1]] = saves
        a[:, 1: saves.shape[1]] *= 2
        Et = torch.fft.ifft(a, dim=1)  # samples in the order of grid.t (Eω = rfft of E on grid.t)
        P = (Et.real ** 2 + Et.imag ** 2) @ self.T.T
        s0 = Il[0].max() if ref_spec is None else ref_spec
        p0 = P[0].max() if ref_env is None else ref_env
        spec = torch.log10(torch.clamp(Il / s0, min=10.0 ** FLOOR))
        return spec.float(), (P / p0).float()


# ----------------------------------------------------------------------------- model
class Ensemble:
    """The MLP ensemble on the GPU: FP32 master weights, BF16 working copies, Adam state
    and the activation buffers of one training batch (torch tensors for the memory)."""

    def __init__(self, members=4, seed=0, batch=4096, lr=1e-3, device="cuda"):
        import torch
        self.torch = torch
        self.members, self.batch, self.lr = members, batch, lr
        self.dev = device
        g = torch.Generator(device="cpu").manual_seed(seed)
        self.fourier = (torch.randn(NFOURIER, NFEAT, generator=g) *
                        torch.logspace(-1.5, 0.7, NFOURIER)[:, None]).to(device)
        self.W, self.b, self.Wb = [], [], []
        self.mW, self.vW, self.mb, self.vb, self.gW, self.gb = [], [], [], [], [], []
        for K, N in zip(WIDTHS[:-1], WIDTHS[1:]):
            W = (torch.randn(members, N, K, generator=g) * math.sqrt(1.0 / K)).to(device)
            self.W.append(W)
            self.b.append(torch.zeros(members, N, device=device))
            self.Wb.append(W.to(torch.bfloat16))
            for lst, like in ((self.mW, W), (self.vW, W), (self.gW, W)):
                lst.append(torch.zeros_like(like))
            for lst in (self.mb, self.vb, self.gb):
                lst.append(torch.zeros(members, N, device=device))
        self.step_no = 0
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self._bufs = {}

    def _buf(self, B, train=True):
        """Buffers for a batch of B: activations and outputs, and for training also the
        pre-activations and gradients."""
        if (B, train) not in self._bufs:
            t = self.torch
            bf = t.bfloat16
            m = self.members
            d = {"feat": t.empty(B, NIN, dtype=bf, device=self.dev),
                 "A": [t.empty(m, B, n, dtype=bf, device=self.dev) for n in WIDTHS[1:-1]],
                 "Y": t.empty(m, B, NOUT, device=self.dev),
                 "loss": t.zeros(m, dtype=t.float64, device=self.dev)}
            if train:
                d["Z"] = [t.empty(m, B, n, dtype=bf, device=self.dev) for n in WIDTHS[1:-1]]
                d["dZ"] = [t.empty(m, B, n, dtype=bf, device=self.dev) for n in WIDTHS[1:]]
            self._bufs[(B, train)] = d
        return self._bufs[(B, train)]

    @staticmethod
    def _p(x):
        return ctypes.c_void_p(x.data_ptr()) if x is not None else None

    def forward(self, x, B=None, keep=True):
        """Outputs [members, B, 768] FP32 for standardised inputs x [B, 8] (FP32 tensor);
        ``keep`` stores the pre-activations a backward pass needs."""
        lib, p = load(), self._p
        B = x.shape[0] if B is None else B
        bf = self._buf(B, keep)
        st = ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)
        _check(lib.luna_sg_features(p(x), B, p(self.fourier), NFOURIER, p(bf["feat"]), NIN, st), "features")
        X, sX = bf["feat"], 0
        nl = len(WIDTHS) - 1
        for l in range(nl):
            K, N = WIDTHS[l], WIDTHS[l + 1]
            last = l == nl - 1
            _check(lib.luna_sg_linear_fwd(p(X), sX, p(self.Wb[l]), p(self.b[l]), B, K, N, 0 if last else 1,
                                          None if last else p(bf["A"][l]),
                                          None if (last or not keep) else p(bf["Z"][l]),
                                          p(bf["Y"]) if last else None, self.members, p(self.err), st), "fwd")
            if not last:
                X, sX = bf["A"][l], B * N
        return bf["Y"]

    def train_step(self, x, T):
        """One Adam step of every member on inputs x [B, 8] and targets T [B, 768] (FP32
        tensors; members share the batch). Returns the mean squared errors [members]."""
        lib, p, t = load(), self._p, self.torch
        B = x.shape[0]
        bf = self._buf(B)
        st = ctypes.c_void_p(t.cuda.current_stream().cuda_stream)
        Y = self.forward(x, B)
        bf["loss"].zero_()
        nl = len(WIDTHS) - 1
        _check(lib.luna_sg_mse(p(Y), p(T), 0, B, NOUT, p(bf["dZ"][nl - 1]), p(bf["loss"]), self.members, st), "mse")
        for l in range(nl - 1, -1, -1):
            K, N = WIDTHS[l], WIDTHS[l + 1]
            Xl, sX = (bf["feat"], 0) if l == 0 else (bf["A"][l - 1], B * K)
            _check(lib.luna_sg_linear_bwd_weight(p(bf["dZ"][l]), p(Xl), sX, B, K, N, p(self.gW[l]), p(self.gb[l]),
                                                 self.members, p(self.err), st), "bwd_weight")
            if l > 0:
                _check(lib.luna_sg_linear_bwd_data(p(bf["dZ"][l]), p(self.Wb[l]), p(bf["Z"][l - 1]), B, K, N,
                                                   p(bf["dZ"][l - 1]), self.members, p(self.err), st), "bwd_data")
        self.step_no += 1
        for l in range(nl):
            _check(lib.luna_sg_adam(p(self.W[l]), p(self.mW[l]), p(self.vW[l]), p(self.gW[l]), self.W[l].numel(),
                                    self.lr, 0.9, 0.999, 1e-8, self.step_no, p(self.Wb[l]), st), "adam")
            _check(lib.luna_sg_adam(p(self.b[l]), p(self.mb[l]), p(self.vb[l]), p(self.gb[l]), self.b[l].numel(),
                                    self.lr, 0.9, 0.999, 1e-8, self.step_no, None, st), "adam")
        return bf["loss"]

    def fold_output_scaling(self, mu, sd):
        """Make the last layer predict sd * y + mu (FP32 master weights and BF16 copy)."""
        self.W[-1] *= sd[None, :, None]
        self.b[-1].mul_(sd[None, :]).add_(mu[None, :])
        self.Wb[-1] = self.W[-1].to(self.torch.bfloat16)

    def predict(self, x):
        """Ensemble mean [B, 768] and spread [B] (largest member standard deviation over the
        spectral outputs, in decades) for standardised inputs x [B, 8]."""
        lib, p, t = load(), self._p, self.torch
        B = x.shape[0]
        Y = self.forward(x, B, keep=False)
        mean = t.empty(B, NOUT, device=self.dev)
        spread = t.empty(B, device=self.dev)
        _check(lib.luna_sg_ensemble(p(Y), self.members, B, NOUT, NSPEC, p(mean), p(spread),
                                    ctypes.c_void_p(t.cuda.current_stream().cuda_stream)), "ensemble")
        return mean, spread

    def check_timeout(self):
        if int(self.err.item()) != 0:
            raise RuntimeError("a tensor-core wait of the surrogate kernels timed out")


def reference_gradients(feat, Wb, b, T, rounding=True):
    """CPU restatement of one member's forward and backward pass (numpy FP64 on the BF16
    inputs and weights the device uses, with activations rounded to BF16 where the device
    stores them; ``rounding=False`` keeps FP64 throughout): the loss and the gradients of
    every W and b, to check the device's."""
    def bf16(a):
        if not rounding:
            return np.asarray(a, dtype=np.float64)
        a = np.asarray(a, dtype=np.float32)
        u = a.view(np.uint32).astype(np.uint64)
        u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
        return u.astype(np.uint32).view(np.float32).astype(np.float64)

    def silu(z):
        return z / (1 + np.exp(-z))

    def dsilu(z):
        s = 1 / (1 + np.exp(-z))
        return s * (1 + z * (1 - s))

    X = [np.asarray(feat, dtype=np.float64)]
    Zs = []
    nl = len(Wb)
    for l in range(nl):
        z = X[-1] @ Wb[l].T + b[l]
        if l == nl - 1:
            Y = z
        else:
            Zs.append(bf16(z))
            X.append(bf16(silu(z)))
    n = Y.size
    loss = float(np.mean((Y - T) ** 2))
    dZ = bf16(2 * (Y - T) / n)
    gW, gb = [None] * nl, [None] * nl
    for l in range(nl - 1, -1, -1):
        gW[l] = dZ.T @ X[l]
        gb[l] = dZ.sum(axis=0)
        if l > 0:
            dZ = bf16((dZ @ Wb[l]) * dsilu(Zs[l - 1]))
    return loss, gW, gb


# ----------------------------------------------------------------------------- data
def draw(n, seed):
    """Seeded draw of the scan family's physical parameters (the ranges of the
    256-instance scan): energy 50-400 µJ, 0.5-5 bar, He/Ne/Ar/H2, radius 75-150 µm,
    τfwhm 8-30 fs."""
    from .scan import GASES as G, RADII
    rng = np.random.default_rng(seed)
    return [dict(energy=float(rng.uniform(50e-6, 400e-6)), pressure=float(rng.uniform(0.5, 5.0)),
                 gas=G[int(rng.integers(0, len(G)))], radius=RADII[int(rng.integers(0, len(RADII)))],
                 τfwhm=float(rng.uniform(8e-15, 30e-15))) for _ in range(n)]


def problem(p, flength=3.0, saveN=201):
    """One data run: the parameters p on the fixed 1 ps, 150 nm - 4 µm grid (8192 samples,
    16384 oversampled), over ``flength`` metres with ``saveN`` saves."""
    from .scan import build_problem
    return build_problem(dict(p, flength=flength, λmin=LAMBDA[0], λmax=LAMBDA[1], trange=1e-12), saveN=saveN)


def generate(params, precision=1, rtol=1e-6, flength=3.0, saveN=201, chunk=256, log=print):
    """Integrate every parameter set with the batched solver (``chunk`` instances per
    persistent launch) and turn the saved fields into targets on the GPU. Returns
    (raw inputs [n, 8], targets [n, 768] FP32 torch tensor, run index [n] of every sample,
    statuses, device seconds)."""
    import torch
    from . import _lib, scan
    from . import plan as P
    probs = [problem(p, flength, saveN) for p in params]
    tg = Targets(probs[0].grid)
    zs = np.linspace(0.0, flength, saveN)
    xs, ts, runs, status, dev_s = [], [], [], [], 0.0
    for c0 in range(0, len(probs), chunk):
        pr = probs[c0:c0 + chunk]
        plans = [P.Plan.from_transform(q.transform, precision) for q in pr]
        b = P.Batch(plans, saveN, zs, rtol=rtol)
        b.upload([q.linop for q in pr], [q.Eω for q in pr], [0.0] * len(pr), [1e-4] * len(pr),
                 [flength] * len(pr), None, [flength / 2] * len(pr))
        b.set_priority([scan.schedule_priority(dict(params[c0 + i], flength=flength), q) for i, q in enumerate(pr)])
        dev_s += b.run() / 1e3
        saves, _, st = b.download()
        for i, (S, s) in enumerate(zip(saves, st)):
            status.append(int(s.status))
            if s.status != 0:
                continue
            spec, env = tg(torch.from_numpy(S).cuda())
            ts.append(torch.cat([spec, env], dim=1))
            q = params[c0 + i]
            xs.append(raw_features([q["energy"]] * saveN, [q["pressure"]] * saveN, [q["radius"]] * saveN,
                                   [q["τfwhm"]] * saveN, zs, [q["gas"]] * saveN))
            runs.append(np.full(saveN, c0 + i))
        del b, plans
        if log:
            log(f"data: {min(c0 + chunk, len(probs))}/{len(probs)} runs, {dev_s:.1f} s of device time")
    return np.concatenate(xs), torch.cat(ts), np.concatenate(runs), status, dev_s


class Standardise:
    def __init__(self, x):
        self.mu = x.mean(axis=0)
        self.sd = np.where(x.std(axis=0) > 0, x.std(axis=0), 1.0)

    def __call__(self, x):
        return (x - self.mu) / self.sd


def train(model, x, T, epochs=40, lr=(1e-3, 1e-5), seed=0, log=print, standardise=True):
    """Adam over shuffled batches of the training set (x: standardised FP32 tensor [n, 8],
    T: FP32 tensor [n, 768]) with a cosine learning-rate decay; returns the loss history.
    With ``standardise`` every output is fitted in units of its spread over the training set
    and the scaling is folded into the last layer afterwards (the trained network then
    predicts the targets' own units)."""
    import torch
    n = x.shape[0]
    mu = sd = None
    if standardise:
        mu = T.mean(dim=0)
        sd = T.std(dim=0).clamp(min=1e-3)
        T = ((T - mu) / sd).contiguous()
    B = model.batch
    steps = epochs * (n // B)
    g = torch.Generator(device="cuda").manual_seed(seed)
    hist = []
    k = 0
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        for s in range(n // B):
            idx = perm[s * B:(s + 1) * B]
            model.lr = lr[1] + 0.5 * (lr[0] - lr[1]) * (1 + math.cos(math.pi * k / max(steps, 1)))
            loss = model.train_step(x[idx].contiguous(), T[idx].contiguous())
            k += 1
        hist.append(loss.cpu().numpy().tolist())
        if log and (ep % max(1, epochs // 8) == 0 or ep == epochs - 1):
            log(f"epoch {ep + 1}/{epochs}: loss per member {np.round(hist[-1], 5).tolist()}")
    model.check_timeout()
    if standardise:
        model.fold_output_scaling(mu, sd)
    return hist


def predict(model, x, chunk=1 << 17):
    """Ensemble mean and spread for standardised inputs x (FP32 tensor [n, 8]); n is padded
    to a multiple of 128 internally."""
    import torch
    n = x.shape[0]
    means, spreads = [], []
    for c0 in range(0, n, chunk):
        xc = x[c0:c0 + chunk]
        m = xc.shape[0]
        pad = (-m) % 128
        if pad:
            xc = torch.cat([xc, xc[:1].expand(pad, -1)])
        mu, sp = model.predict(xc.contiguous())
        means.append(mu[:m])
        spreads.append(sp[:m])
    return torch.cat(means), torch.cat(spreads)


def spectral_error(pred, true):
    """Per point RMS difference of the log10 spectra over the 512 bins (decades)."""
    return ((pred[:, :NSPEC] - true[:, :NSPEC]) ** 2).mean(dim=1).sqrt()


def nearest_neighbour(xtrain, Ttrain, xq, chunk=4096):
    """The method without the network: the target of the nearest training point in the
    standardised input space."""
    import torch
    out = []
    for c0 in range(0, xq.shape[0], chunk):
        d = torch.cdist(xq[c0:c0 + chunk], xtrain)
        out.append(Ttrain[d.argmin(dim=1)])
    return torch.cat(out)
