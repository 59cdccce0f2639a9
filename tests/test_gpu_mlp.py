"""The learned initial guess (svf_mlp_*, SVF_INIT_MLP).  It has no counterpart
in the reference, so its kernels are checked against an FP64 numpy statement
of the same network, and its use against the reference's own path:

* one SGD step equals w - lr * dL/dw of the FP64 network (the backward GEMMs,
  the GELU derivative, the bias column sums), and one Adam step from zero
  moments moves every weight by lr * g / (|g| + 1e-8);
* the features (64 half-vector bins and 32 single pairs of the luminance
  slab) equal their numpy statement, prediction (hidden layers on the tensor
  cores as BF16x3 products with FP32 accumulation, the output layer in FP32)
  equals the FP64 forward pass of the FP32 weights, and the decoded lobe R diag(sx^2, sy^2, 1) R^T equals the
  exponential of the predicted log S with its eigenvalue nearest 0 set to 0;
* a model trained on seeded synthetic texels starts LM fits (with the lighter
  initial damping the learned guess gets by default) of other texels that end,
  texel for texel, at the residual of the fit from the reference's default
  guess on the median and within 10 % of it on average, in fewer iterations,
  with no texel failing;
* save/load round-trips bit-exactly, and svf_fit_btfs with a model matches
  svf_fit_texels with it."""
import struct

import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu

BINS, PAIRS, HIDDEN, OUTPUTS = 64, 32, 256, 8
INPUTS = BINS + PAIRS
W1, B1 = 0, HIDDEN * INPUTS
W2, B2 = B1 + HIDDEN, B1 + HIDDEN + HIDDEN * HIDDEN
W3, B3 = B2 + HIDDEN, B2 + HIDDEN + OUTPUTS * HIDDEN
NPARAMS = B3 + OUTPUTS


def _gelu(x):
    return 0.5 * x * (1 + np.tanh(0.7978845608028654 * (x + 0.044715 * x ** 3)))


def _gelu_grad(x):
    k = 0.7978845608028654
    t = np.tanh(k * (x + 0.044715 * x ** 3))
    return 0.5 * (1 + t) + 0.5 * x * (1 - t * t) * k * (1 + 3 * 0.044715 * x * x)


def _unpack(w):
    w = w.astype(np.float64)
    return (w[W1:B1].reshape(HIDDEN, INPUTS), w[B1:W2], w[W2:B2].reshape(HIDDEN, HIDDEN), w[B2:W3],
            w[W3:B3].reshape(OUTPUTS, HIDDEN), w[B3:])


def _forward(w, X):
    a1, c1, a2, c2, a3, c3 = _unpack(w)
    z1 = X @ a1.T + c1
    h1 = _gelu(z1)
    z2 = h1 @ a2.T + c2
    h2 = _gelu(z2)
    return z1, h1, z2, h2, h2 @ a3.T + c3


def _loss_grad(w, X, T):
    """MSE over all outputs and its gradient, in FP64."""
    a1, c1, a2, c2, a3, c3 = _unpack(w)
    X = X.astype(np.float64)
    z1, h1, z2, h2, y = _forward(w, X)
    n = y.size
    dy = 2 * (y - T) / n
    dh2 = (dy @ a3) * _gelu_grad(z2)
    dh1 = (dh2 @ a2) * _gelu_grad(z1)
    g = np.concatenate([(dh1.T @ X).ravel(), dh1.sum(0), (dh2.T @ h1).ravel(), dh2.sum(0), (dy.T @ h2).ravel(),
                        dy.sum(0)])
    return float(((y - T) ** 2).mean()), g


def _blob(lp, pairs, xmean, xrstd, ymean, ystd, w, features=svf.SVF_MLP_FEATURES_BINS):
    L = lp.shape[0]
    return (b"SVFMLP02" + struct.pack("<III", L, NPARAMS, features) + np.ascontiguousarray(lp, np.float32).tobytes() +
            np.asarray(pairs, np.uint32).tobytes() + np.asarray(xmean, np.float32).tobytes() +
            np.asarray(xrstd, np.float32).tobytes() + np.asarray(ymean, np.float32).tobytes() +
            np.asarray(ystd, np.float32).tobytes() + np.asarray(w, np.float32).tobytes())


def _weights_of(blob):
    return np.frombuffer(blob[-4 * NPARAMS:], np.float32).copy()


def _random_model(lp, seed, scale=0.1):
    rng = np.random.default_rng(seed)
    L = lp.shape[0]
    pairs = rng.choice(L * L, PAIRS, replace=False)
    xmean = rng.normal(-2.0, 0.5, INPUTS)
    xrstd = rng.uniform(0.5, 2.0, INPUTS)
    # outputs around a lobe with well-separated eigenvalues (sx 0.3, sy 0.15, a tilted frame)
    c, s = np.cos(0.4), np.sin(0.4)
    R = np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]]) @ np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])
    logS = R @ np.diag([2 * np.log(0.3), 2 * np.log(0.15), 0]) @ R.T
    ymean = np.array([logS[0, 0], logS[1, 1], logS[2, 2], logS[0, 1], logS[0, 2], logS[1, 2], -1.0, -1.2])
    ystd = np.array([0.1] * 6 + [0.5, 0.5])
    w = rng.normal(0, scale, NPARAMS).astype(np.float32)
    return pairs, xmean, xrstd, ymean, ystd, w


def _bins(lp):
    """The half-vector bins of every direction pair, in the library's FP32 arithmetic."""
    f = np.float32
    lp = np.asarray(lp, f)
    px, py = lp[:, 0], lp[:, 1]
    ls = px * px + py * py
    w = np.stack([f(2) * px / (ls + f(1)), f(2) * py / (ls + f(1)), (f(1) - ls) / (f(1) + ls)], 1)
    h = (w[:, None, :] + w[None, :, :]).reshape(-1, 3)
    n = np.sqrt(h[:, 0] * h[:, 0] + h[:, 1] * h[:, 1] + h[:, 2] * h[:, 2])
    h = h / n[:, None]
    z = f(1) + np.maximum(h[:, 2], f(-0.999))
    hx, hy = h[:, 0] / z, h[:, 1] / z
    r = max(np.abs(hx).max(), np.abs(hy).max(), f(1e-6))
    bx = np.minimum(7, ((hx + r) / (f(2) * r) * f(8)).astype(np.int64))
    by = np.minimum(7, ((hy + r) / (f(2) * r) * f(8)).astype(np.int64))
    return by * 8 + bx


def _features(rgb, lp, pairs):
    """log features [T][96] (not normalised) of RGB samples [T][N][3]."""
    f = np.float32
    lum = (f(0.2126) * rgb[..., 0] + f(0.7152) * rgb[..., 1]) + f(0.0722) * rgb[..., 2]
    b = _bins(lp)
    sums = np.stack([lum[:, b == k].astype(np.float64).mean(1) if (b == k).any() else np.zeros(len(lum))
                     for k in range(BINS)], 1)
    v = np.concatenate([sums, lum[:, pairs].astype(np.float64)], 1)
    return np.log(np.maximum(v, 1e-6))


def _ring(golden):
    m = golden["mesh"]
    return svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])


def test_sgd_and_adam_steps_match_fp64_gradient(gpu_ctx, golden):
    lp = _ring(golden).lights_parabolic
    pairs, xmean, xrstd, ymean, ystd, w = _random_model(lp, 1)
    blob = _blob(lp, pairs, xmean, xrstd, ymean, ystd, w)
    rng = np.random.default_rng(2)
    rows = 200   # ragged against the 64-row tiles
    X = rng.standard_normal((rows, INPUTS)).astype(np.float32)
    T = rng.standard_normal((rows, OUTPUTS)).astype(np.float32)
    loss64, g64 = _loss_grad(w, X, T)

    m = svf.Mlp.load(gpu_ctx, blob)
    assert m.save() == blob
    loss = m.step(X, T, lr=1.0, sgd=True)
    assert loss == pytest.approx(loss64, rel=1e-4)
    g = w.astype(np.float64) - _weights_of(m.save())
    scale = np.abs(g64).max()
    np.testing.assert_allclose(g, g64, atol=2e-4 * scale)
    for name, (a, b) in {"W1": (W1, B1), "b1": (B1, W2), "W2": (W2, B2), "b2": (B2, W3), "W3": (W3, B3),
                         "b3": (B3, NPARAMS)}.items():
        err = np.abs(g[a:b] - g64[a:b]).max() / np.abs(g64[a:b]).max()
        assert err < 2e-3, (name, err)
    m.close()

    # Adam from zero moments: the bias-corrected step is lr * g / (|g| + 1e-8)
    m = svf.Mlp.load(gpu_ctx, blob)
    lr = 1e-3
    m.step(X, T, lr=lr, sgd=False)
    d = (w.astype(np.float64) - _weights_of(m.save())) / lr
    # (where |g| is within a few decades of the 1e-8 the FP32 gradient's own error
    # moves g / (|g| + 1e-8) visibly: those weights are only held to |step| <= lr)
    big = np.abs(g64) >= 1e-6
    np.testing.assert_allclose(d[big], (g64 / (np.abs(g64) + 1e-8))[big], atol=2e-3)
    assert np.abs(d).max() <= 1.0 + 1e-3
    m.close()


def test_predict_matches_fp64_forward(gpu_ctx, oracle_lib, golden):
    lp = _ring(golden).lights_parabolic
    pairs, xmean, xrstd, ymean, ystd, w = _random_model(lp, 3, scale=0.05)
    m = svf.Mlp.load(gpu_ctx, _blob(lp, pairs, xmean, xrstd, ymean, ystd, w))
    T = 300
    rgb = np.stack([oracle_lib.synth_render(9, x, oracle_lib.synth_truth(9, 1, x), lp) for x in range(T)])
    rgb[0, pairs[0], :] = 0.0   # the log clamp at 1e-6
    p, feats = m.predict(rgb, T, features=True)
    x64 = (_features(rgb, lp, pairs) - xmean) * xrstd
    np.testing.assert_allclose(feats, x64, rtol=1e-5, atol=1e-4)
    # the FP64 network on the FP32 weights: the split products carry 16
    # significant bits of each operand, so the outputs agree to ~1e-5 relative
    y = _forward(w.astype(np.float64), feats.astype(np.float64))[-1] * ystd + ymean
    np.testing.assert_allclose(p[:, 2], np.maximum(np.exp(y[:, 6]) - 1e-4, 0), rtol=1e-4, atol=1e-7)
    np.testing.assert_allclose(p[:, 3], np.maximum(np.exp(y[:, 7]) - 1e-4, 0), rtol=1e-4, atol=1e-7)
    assert (p[:, 0] >= p[:, 1]).all()
    for t in range(T):
        M = np.array([[y[t, 0], y[t, 3], y[t, 4]], [y[t, 3], y[t, 1], y[t, 5]], [y[t, 4], y[t, 5], y[t, 2]]])
        lam, V = np.linalg.eigh(M)
        lam[np.argmin(np.abs(lam))] = 0.0
        S64 = V @ np.diag(np.minimum(np.exp(lam / 2), 4) ** 2) @ V.T
        R, _ = oracle_lib.euler_to_matrix(p[t, 4:7])   # R[c] is column c
        S = p[t, 0] ** 2 * np.outer(R[0], R[0]) + p[t, 1] ** 2 * np.outer(R[1], R[1]) + np.outer(R[2], R[2])
        np.testing.assert_allclose(S, S64, atol=2e-3)
    # device samples give the same prediction
    import torch

    p2 = m.predict(torch.from_numpy(rgb).cuda(), T)
    np.testing.assert_array_equal(p, p2)
    m.close()
    # the other feature set: the 32 pairs' RGB samples, log-scaled
    m = svf.Mlp.load(gpu_ctx, _blob(lp, pairs, xmean, xrstd, ymean, ystd, w, svf.SVF_MLP_FEATURES_PAIRS_RGB))
    _, f_rgb = m.predict(rgb, T, features=True)
    x_rgb = (np.log(np.maximum(rgb[:, pairs, :].reshape(T, INPUTS).astype(np.float64), 1e-6)) - xmean) * xrstd
    np.testing.assert_allclose(f_rgb, x_rgb, rtol=1e-5, atol=1e-4)
    m.close()


def test_model_checks(gpu_ctx, golden):
    lp = _ring(golden).lights_parabolic
    model = _random_model(lp, 4)
    blob = _blob(lp, *model)
    with pytest.raises(svf.SvfError):
        svf.Mlp.load(gpu_ctx, blob[:-4])
    with pytest.raises(svf.SvfError):
        svf.Mlp.load(gpu_ctx, b"XXXXXXXX" + blob[8:])
    with pytest.raises(svf.SvfError):   # unknown feature set
        svf.Mlp.load(gpu_ctx, _blob(lp, *model, features=7))
    bad_pairs = np.array(model[0])
    bad_pairs[3] = 81 * 81
    with pytest.raises(svf.SvfError):
        svf.Mlp.load(gpu_ctx, _blob(lp, bad_pairs, *model[1:]))
    # a model of the ring layout on a Fibonacci-layout BTF
    m = svf.Mlp.load(gpu_ctx, blob)
    lp151 = svf.directions_fibonacci(151)
    fib = svf.Layout(lp151, *svf.triangulate(lp151))
    with pytest.raises(svf.SvfError):
        gpu_ctx.fit_texels(fib, np.zeros((2, 151 * 151, 3), np.float32), 2, 1, mlp=m, want=("rmse",))
    assert "another direction layout" in svf.load().svf_last_error().decode()
    m.close()


@pytest.fixture(scope="module")
def trained(gpu_ctx, golden):
    lp = _ring(golden).lights_parabolic
    m, loss = svf.Mlp.train(gpu_ctx, lp, svf.mlp_train_options(texels=1 << 18, epochs=12, batch=2048, seed=77))
    yield m, loss
    m.close()


def test_trained_model_starts_fits_at_the_default_guess_residual(gpu_ctx, golden, trained):
    import torch

    m, loss = trained
    assert np.isfinite(loss) and loss < 0.25, loss   # of the normalised targets' unit variance
    lay = _ring(golden)
    T = 8192
    s = torch.empty((T, 81 * 81, 3), dtype=torch.float32, device="cuda")
    gpu_ctx.synth_btf(2031, 1, lay.lights_parabolic, 0, T, s)   # texels the model never saw
    ref, rs0 = gpu_ctx.fit_texels(lay, s, 128, 64, want=("rmse", "params", "stats"))
    got, rs1 = gpu_ctx.fit_texels(lay, s, 128, 64, mlp=m, want=("rmse", "params", "init", "stats"))
    assert rs1.failed_texels == 0
    np.testing.assert_array_equal(got["init"], m.predict(s, T))
    ratio = got["rmse"] / ref["rmse"]
    stats = dict(median=np.median(ratio), within=np.mean(ratio <= 1.01), mean_rmse=got["rmse"].mean(),
                 ref_mean_rmse=ref["rmse"].mean(), iters=got["stats"]["iterations"].mean(),
                 ref_iters=ref["stats"]["iterations"].mean())
    assert stats["median"] <= 1.001, stats
    assert stats["within"] >= 0.6, stats
    # the mean is carried by the few texels the guess sends into another local
    # minimum (what the plain-LM fallback catches): within 10 %
    assert stats["mean_rmse"] <= 1.10 * stats["ref_mean_rmse"], stats
    assert stats["iters"] < stats["ref_iters"], stats
    # the reference's damping from the learned guess: the early stop the lighter start avoids
    full, _ = gpu_ctx.fit_texels(lay, s, 128, 64, mlp=m, damping=1.0, want=("rmse",))
    assert full["rmse"].mean() > stats["mean_rmse"], (full["rmse"].mean(), stats)


def test_save_load_and_batch_with_a_model(gpu_ctx, golden, trained, oracle_lib):
    m, _ = trained
    lay = _ring(golden)
    lp = lay.lights_parabolic
    m2 = svf.Mlp.load(gpu_ctx, m.save())
    assert m2.save() == m.save()
    a = np.stack([oracle_lib.synth_render(5, x, oracle_lib.synth_truth(5, 1, x), lp) for x in range(40)])
    b = np.stack([oracle_lib.synth_render(6, x, oracle_lib.synth_truth(6, 1, x), lp) for x in range(24)])
    np.testing.assert_array_equal(m.predict(a, 40), m2.predict(a, 40))
    want = ("params", "rmse", "init")
    with svf.Context(0) as ctx:
        maps, runs, total = ctx.fit_btfs([dict(layout=lay, samples=a, width=8, height=5, mlp=m),
                                          dict(layout=lay, samples=b, width=6, height=4)], want=want)
        assert total.failed_texels == 0
        alone, _ = ctx.fit_texels(lay, a, 8, 5, mlp=m, want=want)
        for k in want:
            np.testing.assert_array_equal(maps[0][k], alone[k], err_msg=k)
        # the RGB fit chains from the luminance fit of the learned guess
        rgb, _ = ctx.fit_texels(lay, a, 8, 5, mlp=m, opts=svf.options(rgb=True), want=("rmse",))
        col, _ = ctx.fit_texels(lay, a, 8, 5, mlp=m, want=("diffuse", "specular", "sigma", "basis"))
        start = np.concatenate([col["diffuse"], col["specular"], col["sigma"], col["basis"]], 1)
        base, _ = ctx.fit_texels(lay, a, 8, 5, opts=svf.options(rgb=True, max_iterations=0), init=start,
                                 want=("rmse",))
        assert (rgb["rmse"] <= base["rmse"] * (1 + 1e-6)).all()
    m2.close()


def test_plain_lm_fallback(gpu_ctx, golden, trained):
    """SVF_INIT_MLP with mlp_fallback: texels whose RMSE from the learned guess is
    above the threshold (relative to their luminance slice's RMS) are fitted from
    the default guess as well and keep the lower RMSE; the others keep the
    learned-guess fit.  Both fits are the ones the two modes give alone, bit for
    bit, so the result is their per-texel minimum where selected."""
    import torch

    m, _ = trained
    lay = _ring(golden)
    W, H = 64, 64
    T = W * H
    s = torch.empty((T, 81 * 81, 3), dtype=torch.float32, device="cuda")
    gpu_ctx.synth_btf(4040, 1, lay.lights_parabolic, 0, T, s)
    want = ("rmse", "params", "diffuse", "basis")
    plain, _ = gpu_ctx.fit_texels(lay, s, W, H, want=want)
    learned, _ = gpu_ctx.fit_texels(lay, s, W, H, mlp=m, want=want)
    x = s.cpu().numpy()
    lum = (np.float32(0.2126) * x[..., 0] + np.float32(0.7152) * x[..., 1]) + np.float32(0.0722) * x[..., 2]
    rel = learned["rmse"] / np.sqrt((lum.astype(np.float64) ** 2).mean(1))
    th = float(np.median(rel))
    got, rs = gpu_ctx.fit_texels(lay, s, W, H, mlp=m, fallback=th, want=want)
    assert rs.failed_texels == 0
    above, below = rel > th * (1 + 1e-5), rel < th * (1 - 1e-5)
    assert above.sum() <= rs.fallback_texels <= T - below.sum()
    best = np.minimum(learned["rmse"], plain["rmse"])
    np.testing.assert_array_equal(got["rmse"][above], best[above])
    np.testing.assert_array_equal(got["rmse"][below], learned["rmse"][below])
    take = above & (plain["rmse"] < learned["rmse"])
    for k in ("params", "diffuse", "basis"):
        np.testing.assert_array_equal(got[k][take], plain[k][take], err_msg=k)
        np.testing.assert_array_equal(got[k][below], learned[k][below], err_msg=k)
    assert (got["rmse"] <= learned["rmse"]).all()
    with pytest.raises(svf.SvfError):   # the fallback belongs to the learned guess
        gpu_ctx.fit_texels(lay, s, W, H, fallback=0.5, want=("rmse",))
