"""Schedule layer on the GPU: the MLP kernels against a NumPy restatement
(forward and gradient), training, model-chosen windows, the exhaustive
autotuner and the scalar histogram."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _np_grad(params, X, t, w=None):
    """Analytic gradient of the (weighted) batch MSE for the kernel's parameter
    layout."""
    w = np.ones(X.shape[0]) if w is None else w
    D, H1, H2 = X.shape[1], 64, 64
    sizes = [D * H1, H1, H1 * H2, H2, H2, 1]
    offs = np.cumsum([0] + sizes)
    W1 = params[offs[0]:offs[1]].reshape(D, H1)
    b1 = params[offs[1]:offs[2]]
    W2 = params[offs[2]:offs[3]].reshape(H1, H2)
    b2 = params[offs[3]:offs[4]]
    W3 = params[offs[4]:offs[5]]
    b3 = params[offs[5]]
    z1 = X @ W1 + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2 + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ W3 + b3
    B = X.shape[0]
    g = 2 * w * (y - t) / B
    dW3 = h2.T @ g
    db3 = g.sum()
    d2 = np.outer(g, W3) * (z2 > 0)
    dW2 = h1.T @ d2
    db2 = d2.sum(0)
    d1 = (d2 @ W2.T) * (z1 > 0)
    dW1 = X.T @ d1
    db1 = d1.sum(0)
    loss = np.mean(w * (y - t) ** 2)
    return np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3, [db3]]), loss, y


def test_mlp_forward_and_gradient(gpu):
    S = gpu.schedule
    L = gpu.load_library()
    D = L.zkp_mlp_input_dim()
    m = S.Model.fresh(seed=3)
    rng = np.random.default_rng(0)
    B = 257
    X = rng.normal(size=(B, D)).astype(np.float32)
    t = rng.normal(size=B).astype(np.float32)
    p = m.params.cpu().numpy().astype(np.float64)
    wts = rng.uniform(0.2, 3.0, size=B).astype(np.float32)
    xd, td, wd = torch.from_numpy(X).cuda(), torch.from_numpy(t).cuda(), torch.from_numpy(wts).cuda()
    for w in (None, wts):
        g_np, loss_np, y_np = _np_grad(p, X.astype(np.float64), t.astype(np.float64),
                                       None if w is None else w.astype(np.float64))
        assert np.allclose(m.predict(X), y_np, rtol=1e-4, atol=1e-4)
        assert np.allclose(S.mlp_forward_numpy(p, X.astype(np.float64)), y_np)
        grads = torch.empty_like(m.params)
        loss = torch.zeros(1, dtype=torch.float32, device="cuda")
        scratch = torch.empty(L.zkp_mlp_scratch_floats(B), dtype=torch.float32, device="cuda")
        gpu.abi.check(L.zkp_mlp_grad(m.params.data_ptr(), xd.data_ptr(), td.data_ptr(),
                                     None if w is None else wd.data_ptr(), B, grads.data_ptr(), loss.data_ptr(),
                                     scratch.data_ptr(), gpu.host.stream_handle()))
        g = grads.cpu().numpy()
        assert abs(float(loss.item()) - loss_np) <= 1e-4 * max(1.0, loss_np)
        # FP32 kernel vs float64 NumPy: tolerance 1e-4 relative to the gradient norm
        assert np.max(np.abs(g - g_np)) <= 1e-4 * max(1.0, np.max(np.abs(g_np)))


def test_mlp_training_fits(gpu):
    S = gpu.schedule
    rng = np.random.default_rng(1)
    D = gpu.load_library().zkp_mlp_input_dim()
    X = rng.uniform(-1, 1, size=(512, D)).astype(np.float32)
    y = (np.sin(2 * X[:, 0]) + X[:, -1] ** 2 - 0.5 * X[:, 3]).astype(np.float32)
    m = S.Model.fresh(seed=5)
    hist = m.train(X, y, steps=2000, lr=3e-3)
    assert hist[-1][1] < 0.1 * hist[0][1]
    # model-chosen window == argmin of the model over the candidates
    feats = list(X[0, :D - 1])
    cands = list(range(8, 21))
    pred = m.predict(np.array([feats + [(c - 12) / 8.0] for c in cands], np.float32))
    assert m.pick(feats, 8, 20) == cands[int(np.argmin(pred))]


def test_scalar_histogram(O, gpu):
    S = gpu.schedule
    n = 5000
    for mix in S.MIXES:
        s = S.scalars(n, mix, 11)
        h = S.histogram(s)
        vals = O.fr_ints(gpu.host.to_host(s))
        bins = [0] * 7
        for v in vals:
            b = v.bit_length()
            bins[0 if b == 0 else 1 if b <= 16 else 2 if b <= 32 else 3 if b <= 64 else 4 if b <= 128 else
                 5 if b <= 192 else 6] += 1
        assert np.allclose(h, np.array(bins) / n)
        if mix == "small":
            assert all(v < (1 << 20) for v in vals)


def test_autotune_picks_fastest_and_is_exact(O, gpu):
    S = gpu.schedule
    n = 1 << 14
    bases, k = S.bases_with_known_logs(n, 21)
    s = S.scalars(n, "mixed", 22)
    best, times = S.autotune(bases, s, n, 8, 16, reps=1)
    assert best == min(times, key=times.get)
    # every window gives the same point
    H = gpu.host
    dl = O.fr_vec([int(x) for x in k.cpu().numpy()])
    exp = O.msm_known_dlog(dl, H.to_host(s))
    for c in (8, best, 16):
        out = H.msm(bases, s, n=n, window_bits=c)
        torch.cuda.synchronize()
        assert (O.g1_jac_to_aff(H.to_host(out).reshape(1, 12)) == exp).all()


def test_autotune_extend_small(gpu):
    # the extend-phase search covers both table layouts and the chunk sizes
    best, times = gpu.schedule.autotune_extend(14, 2, 4, chunks=(2, 4), reps=1)
    assert set(times) == {("montgomery", 2), ("pairs", 2), ("montgomery", 4), ("pairs", 4)}
    assert best in times
