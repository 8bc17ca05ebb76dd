"""The predictor network: the CPU oracle (oracle/mlp_oracle.py) pinned by
finite differences, and the GPU forward/backward/Adam kernels
(zerork_b200/csrc/mlp.cu) checked against the oracle.

GPU tolerances: products accumulate in FP32 on the GPU and FP64 in the
oracle, which only moves BF16 roundings of the intermediate values; every
gradient tensor must agree within 1e-2 relative (L2) and every output within
1e-2 of the output scale.
"""
import numpy as np
import pytest

import mlp_oracle as mo
from conftest import have_gpu


def _net(rng, n_in, hidden, layers, n_out):
    d = mo.dims(n_in, hidden, layers, n_out)
    w = np.concatenate([
        (rng.standard_normal((d[l], d[l + 1])) / np.sqrt(d[l])).astype(np.float32).ravel()
        for l in range(len(d) - 1)])
    b = (0.1 * rng.standard_normal(sum(d[1:]))).astype(np.float32)
    # zero the padding rows/columns, as the library keeps them
    W, B = mo.unpack(w, b, d)
    for l, Wl in enumerate(W):
        kin = n_in if l == 0 else hidden
        kout = n_out if l == len(W) - 1 else hidden
        Wl[kin:, :] = 0.0
        Wl[:, kout:] = 0.0
        B[l][kout:] = 0.0
    return d, w, b


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5, 3.0e-39, 65504.0], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0078125)
    assert r[3] == -2.5
    assert np.all(np.isfinite(r))


def test_oracle_gradient_matches_finite_differences(monkeypatch):
    rng = np.random.default_rng(1)
    monkeypatch.setattr(mo, "bf16", lambda a: np.asarray(a, np.float32))  # exact arithmetic
    d, w, b = _net(rng, 7, 16, 2, 5)
    x = rng.standard_normal((32, 7)).astype(np.float32)
    t = rng.standard_normal((32, 5))
    _, gw, gb, _ = mo.forward_backward(w, b, d, x, t)
    n, n_out = t.shape
    for idx in rng.choice(np.flatnonzero(w), 12, replace=False):
        e = 1e-3
        wp, wm = w.copy(), w.copy()
        wp[idx] += e
        wm[idx] -= e
        lp = mo.forward_backward(wp, b, d, x, t)[0] / (n * n_out)
        lm = mo.forward_backward(wm, b, d, x, t)[0] / (n * n_out)
        assert abs((lp - lm) / (2 * e) - gw[idx]) <= 2e-3 * max(1e-3, abs(gw[idx]))
    for idx in rng.choice(np.flatnonzero(b), 6, replace=False):
        e = 1e-3
        bp, bm = b.copy(), b.copy()
        bp[idx] += e
        bm[idx] -= e
        lp = mo.forward_backward(w, bp, d, x, t)[0] / (n * n_out)
        lm = mo.forward_backward(w, bm, d, x, t)[0] / (n * n_out)
        assert abs((lp - lm) / (2 * e) - gb[idx]) <= 2e-3 * max(1e-3, abs(gb[idx]))


@pytest.fixture(scope="module")
def torch():
    if not have_gpu():
        pytest.skip("no CUDA device")
    import torch
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("n_in,n_out,batch", [(163, 161, 64), (14, 12, 48)])
def test_gpu_gradients_match_oracle(torch, n_in, n_out, batch):
    from zerork_b200.predictor import Mlp
    rng = np.random.default_rng(2)
    net = Mlp(n_in, n_out, 256, 3, seed=3)
    d = mo.dims(n_in, 256, 3, n_out)
    _, w, b = _net(rng, n_in, 256, 3, n_out)
    net.set_params(w, b)
    x = rng.standard_normal((batch, n_in)).astype(np.float32)
    t = rng.standard_normal((batch, n_out)).astype(np.float32)
    xd, td = torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda()
    loss = torch.zeros(1, dtype=torch.float32, device="cuda")
    net.gradients(xd, td, loss)
    gw, gb = net.grads()
    y = net.forward(xd).cpu().numpy()
    lo, ow, ob, yo = mo.forward_backward(w, b, d, x, t.astype(np.float64))
    scale = np.abs(yo).max()
    assert np.max(np.abs(y - yo)) <= 1e-2 * scale
    assert abs(float(loss.item()) - lo) <= 1e-2 * lo
    W, B = mo.unpack(gw, gb, d)
    Wo, Bo = mo.unpack(ow, ob, d)
    for l in range(len(W)):
        for g, go in ((W[l], Wo[l]), (B[l], Bo[l])):
            rel = np.linalg.norm(g - go) / max(np.linalg.norm(go), 1e-30)
            assert rel <= 1e-2, (l, rel)


@pytest.mark.gpu
def test_gpu_training_reduces_loss(torch):
    from zerork_b200.predictor import train
    rng = np.random.default_rng(4)
    A = rng.standard_normal((10, 6))
    x = rng.standard_normal((16384, 10))
    t = np.tanh(0.5 * (x @ A)) + 0.1 * (x[:, :6] ** 2)
    net, xs, ts, hist = train(x, t, hidden=256, layers=3, epochs=8, batch=1024, lr=2e-3)
    assert hist[-1] < 0.2 * hist[0], hist
    # the trained network predicts held-out points of the same function
    xv = rng.standard_normal((2048, 10))
    tv = np.tanh(0.5 * (xv @ A)) + 0.1 * (xv[:, :6] ** 2)
    yv = net.forward(torch.from_numpy(xs.fwd(xv).astype(np.float32)).cuda()).cpu().numpy()
    err = np.mean((ts.inv(yv) - tv) ** 2) / np.var(tv)
    assert err < 0.3, err
