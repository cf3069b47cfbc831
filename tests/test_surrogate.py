"""The learned surrogate's kernels (luna.jl_b200/csrc/surrogate.cu) and its training.

* the three tensor-core products of a linear layer against torch's FP32 matmul of the same
  BF16 operands (FP32 accumulation in both);
* one training step's gradients against the CPU restatement (numpy FP64 on the device's
  BF16 operands, ``surrogate.reference_gradients``): relative L2 <= 2e-2 per tensor (BF16
  rounding of the stored activations and gradients);
* training on solver data: the loss falls, and on held-out runs the network's log-spectrum
  error is below that of the method without it (the nearest training point) while it
  answers queries more than 1000x faster than the solver integrates them.
"""
import ctypes
import time

import luna_b200_loader  # registers the luna.jl_b200 package

luna_b200_loader.load()

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from luna_b200 import surrogate as S  # noqa: E402


def _p(t):
    return ctypes.c_void_p(t.data_ptr())


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("B,K,N,members", [(256, 256, 512, 2), (128, 512, 768, 1), (384, 512, 256, 3)])
def test_linear_layer_products_match_matmul(B, K, N, members):
    lib = S.load()
    g = torch.Generator(device="cuda").manual_seed(B + K + N)
    X = torch.randn(members, B, K, device="cuda", generator=g).to(torch.bfloat16)
    W = (torch.randn(members, N, K, device="cuda", generator=g) / K ** 0.5).to(torch.bfloat16)
    b = torch.randn(members, N, device="cuda", generator=g)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    Yf = torch.empty(members, B, N, device="cuda")
    Z = torch.empty(members, B, N, device="cuda", dtype=torch.bfloat16)
    assert lib.luna_sg_linear_fwd(_p(X), B * K, _p(W), _p(b), B, K, N, 0, None, _p(Z), _p(Yf), members, _p(err), st) == 0
    ref = torch.bmm(X.float(), W.float().transpose(1, 2)) + b[:, None, :]
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert _rel(Yf.cpu(), ref.cpu()) < 1e-5
    assert _rel(Z.float().cpu(), ref.cpu()) < 5e-3
    # backward data with the SiLU derivative of a previous layer's pre-activation
    dZ = torch.randn(members, B, N, device="cuda", generator=g).to(torch.bfloat16)
    Zp = torch.randn(members, B, K, device="cuda", generator=g).to(torch.bfloat16)
    dX = torch.empty(members, B, K, device="cuda", dtype=torch.bfloat16)
    assert lib.luna_sg_linear_bwd_data(_p(dZ), _p(W), _p(Zp), B, K, N, _p(dX), members, _p(err), st) == 0
    s = torch.sigmoid(Zp.float())
    ref = torch.bmm(dZ.float(), W.float()) * (s * (1 + Zp.float() * (1 - s)))
    torch.cuda.synchronize()
    assert _rel(dX.float().cpu(), ref.cpu()) < 5e-3
    # backward weights and bias
    dW = torch.empty(members, N, K, device="cuda")
    db = torch.empty(members, N, device="cuda")
    assert lib.luna_sg_linear_bwd_weight(_p(dZ), _p(X), B * K, B, K, N, _p(dW), _p(db), members, _p(err), st) == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert _rel(dW.cpu(), torch.bmm(dZ.float().transpose(1, 2), X.float()).cpu()) < 1e-5
    assert _rel(db.cpu(), dZ.float().sum(dim=1).cpu()) < 1e-5


def test_training_step_gradients_match_cpu_reference():
    m = S.Ensemble(members=2, seed=3, batch=128)
    g = torch.Generator(device="cuda").manual_seed(9)
    x = torch.randn(128, S.NFEAT, device="cuda", generator=g)
    T = torch.randn(128, S.NOUT, device="cuda", generator=g) * 0.5
    Wb = [w.float().cpu().numpy().astype(np.float64) for w in m.Wb]
    bb = [b.cpu().numpy().astype(np.float64) for b in m.b]
    loss = m.train_step(x, T)
    torch.cuda.synchronize()
    m.check_timeout()
    feat = m._buf(128)["feat"].float().cpu().numpy()
    Tn = T.cpu().numpy().astype(np.float64)
    for z in range(2):
        lref, gW, gb = S.reference_gradients(feat, [w[z] for w in Wb], [b[z] for b in bb], Tn)
        assert abs(float(loss[z]) / lref - 1) < 1e-3
        for l in range(len(gW)):
            assert _rel(m.gW[l][z].cpu().numpy(), gW[l]) < 2e-2, (z, l)
            assert _rel(m.gb[l][z].cpu().numpy(), gb[l]) < 2e-2, (z, l)


def test_surrogate_trained_on_solver_data_beats_the_method_without_it():
    """96 runs of 0.5 m (51 saves each) from the batched solver, 80 for training and 16
    held out; 60 epochs."""
    params = S.draw(96, seed=5)
    t0 = time.perf_counter()
    xr, T, runs, status, dev_s = S.generate(params, flength=0.5, saveN=51, chunk=96, log=None)
    solve_s = time.perf_counter() - t0
    ok_runs = sorted(set(runs.tolist()))
    held = set(ok_runs[-16:])
    tr = np.array([r not in held for r in runs])
    std = S.Standardise(xr[tr])
    x = torch.tensor(std(xr), dtype=torch.float32, device="cuda")
    trm = torch.from_numpy(tr).cuda()
    model = S.Ensemble(members=4, seed=1, batch=512)
    hist = S.train(model, x[trm].contiguous(), T[trm].contiguous(), epochs=60, log=None)
    assert np.mean(hist[-1]) < 0.2 * np.mean(hist[0])
    xq, Tq = x[~trm].contiguous(), T[~trm].contiguous()
    mean, spread = S.predict(model, xq)
    # query throughput on 65536 points (the held-out inputs repeated)
    xb = xq.repeat((65536 + xq.shape[0] - 1) // xq.shape[0], 1)[:65536].contiguous()
    S.predict(model, xb, chunk=65536)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    S.predict(model, xb, chunk=65536)
    torch.cuda.synchronize()
    q_s = (time.perf_counter() - t1) / xb.shape[0]
    e_net = float(S.spectral_error(mean, Tq).mean())
    e_nn = float(S.spectral_error(S.nearest_neighbour(x[trm], T[trm], xq), Tq).mean())
    assert e_net < e_nn, (e_net, e_nn)
    # the solver's time per query point: its wall time per run over the points a run saves
    solver_q_s = solve_s / len(params) / 51
    assert solver_q_s / q_s > 1000, (solver_q_s, q_s)
    assert torch.isfinite(spread).all()
