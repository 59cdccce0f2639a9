"""The pseudo-volume multi-scattering BRDF (svbrdffit -m) on the GPU
(svf_ms.cu): the fit's evaluator and svf_render_btf_ms against the reference's
values (tests/golden/ref_ms.npz) and the oracle's restatement (bit-exact to the
reference, tests/test_oracle_ms.py), and the SVF_LSQ_MULTI_SCATTERING fit
against the reference's LeastSquaresFitSGGX with MultiScatteringBounceCount.

The GPU rounds every float operation as the reference does (svf_ms.cu is built
without fused multiply-adds); its logf, expf and tanf differ from glibc's in the
last bits.  A walk sums those differences (about 1e-6 relative), except where
they move a value across one of its break tests, which changes the rest of that
walk and the random numbers of the walks after it: such a pair is a different
Monte Carlo estimate of the same integral.  The bars: 99 % of the values within
1e-4 relative, every value within 25 % (the estimator's spread at 256 walks).
"""
import os

import numpy as np
import pytest

import oracle
import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ms():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_ms.npz"))


def _close(got, ref, where):
    rel = np.abs(got.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-6)
    assert np.mean(rel <= 1e-4) >= 0.99, (where, np.mean(rel <= 1e-4), rel.max())
    assert rel.max() <= 0.25, (where, rel.max())
    return rel


def test_fit_evaluator_matches_reference(gpu_ctx, ms):
    """The RMSE of a zero-iteration fit is the RMS of (slice - model): against the
    reference's own model values it is the evaluation difference, against zeros
    the model's RMS."""
    for i, p in enumerate(ms["params"]):
        for j, b in enumerate(ms["bounces"]):
            ref = ms["brdf_fib32"][i, j]
            opts = svf.options(max_iterations=0, multi_scattering=int(b))
            lum = np.stack([ref, np.zeros_like(ref)]).astype(np.float32)
            init = np.stack([p, p]).astype(np.float32)
            out, rmse, st = gpu_ctx.lsq_fit_batch(ms["fib32"], lum, init, opts)
            assert np.array_equal(out, init) and (st["iterations"] == 0).all()
            rms = float(np.sqrt(np.mean(ref.astype(np.float64) ** 2)))
            np.testing.assert_allclose(rmse[1], rms, rtol=1e-4)
            assert rmse[0] <= 2e-3 * rms, (i, int(b), rmse[0], rms)


def test_render_matches_oracle_rgb(gpu_ctx, ms):
    """svf_render_btf_ms against the oracle's pseudo-volume BRDF in RGB (the walk
    stops when any channel's throughput falls to 1e-3), pair by pair."""
    rng = np.random.default_rng(3)
    lp = ms["fib32"]
    L = lp.shape[0]
    T = 3
    q = rng.standard_normal((T, 4)).astype(np.float32)
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    sigma = (0.05 + 0.4 * rng.random((T, 2))).astype(np.float32)
    diffuse = (0.3 * rng.random((T, 3))).astype(np.float32)
    specular = (0.2 + 1.5 * rng.random((T, 3))).astype(np.float32)
    for bounces in (1, 3):
        got = gpu_ctx.render_btf_ms(lp, diffuse, specular, sigma, q, bounces)
        for t in range(T):
            prm = np.concatenate([sigma[t], q[t], diffuse[t], specular[t]]).astype(np.float32)
            ref = np.stack([oracle.pseudo_volume_rgb(prm, lp, k // L, k % L, bounces) for k in range(L * L)])
            _close(got[t], ref, (t, bounces))


def test_render_evaluator_seed_matches_fit_model(gpu_ctx, ms):
    """With grey albedos, 256 walks and seed 0 the render is the fit's model: the
    reference's evaluator values of params[0] on ring-81 (quaternion from the Euler
    angles as the reference forms it)."""
    p = ms["params"][0].astype(np.float32)
    lp = ms["ring81"]
    e = p[4:].astype(np.float64) * 0.5
    s, c = np.sin(e), np.cos(e)
    quat = np.array([s[0] * c[1] * c[2] + c[0] * s[1] * s[2], -s[0] * c[1] * s[2] + c[0] * s[1] * c[2],
                     c[0] * c[1] * s[2] + s[0] * s[1] * c[2], c[0] * c[1] * c[2] - s[0] * s[1] * s[2]], np.float32)
    got = gpu_ctx.render_btf_ms(lp, np.full((1, 3), p[3], np.float32), np.full((1, 3), p[2], np.float32),
                                p[None, :2], quat[None], 2)
    ref = ms["brdf_ring81"]
    for c_ in range(3):
        # the quaternion above rounds differently from the reference's FastSinCos:
        # the bar is the statistical one, with a looser value bar
        rel = np.abs(got[0, :, c_].astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-6)
        assert np.median(rel) <= 1e-4 and np.mean(rel <= 1e-3) >= 0.95, (c_, np.median(rel), rel.max())


def test_fit_against_reference_goldens(gpu_ctx, ms):
    """SVF_LSQ_MULTI_SCATTERING against the reference's LeastSquaresFitSGGX with
    MultiScatteringBounceCount 2 on the golden slices (16 directions, 6 texels)."""
    opts = svf.options(multi_scattering=int(ms["fit_bounces"]))
    out, rmse, st = gpu_ctx.lsq_fit_batch(ms["fib16"], ms["fit_lum"], ms["fit_init"], opts)
    assert (st["status"] == 0).all()
    ratio = rmse / ms["fit_rmse"]
    # the GPU's evaluations differ from the reference's in the last bits, and the
    # LM from a perturbed start is sensitive to them: most texels end where the
    # reference does, none much above it (the parameters of equal residuals can
    # differ: the diffuse albedo of a strong lobe is barely determined)
    assert np.mean(ratio <= 1.01) >= 0.66 and ratio.max() <= 1.25, ratio


def test_fit_against_oracle(gpu_ctx):
    """16 texels of the uneven mix on the 16-direction layout, bounces 1 and 3:
    the GPU fit against the oracle's (the reference's LM and model, bit-exact).

    From a perturbed start the reference's LM on this model is chaotic in the last
    bits of its evaluations: the oracle itself, with logf moved by one ulp, ends
    within 1 % of its own fit on 16/16 of these texels at 1 bounce but on 11/16 at
    3 bounces, with three texels at 1.4 - 1.7 x (measured).  The bars follow that
    spread: at 1 bounce most texels agree, at 3 the median does."""
    lp = svf.directions_fibonacci(16)
    rng = np.random.default_rng(17)
    T = 16
    for bounces in (1, 3):
        truth, lum, init = [], [], []
        for _ in range(T):
            p = np.array([0.05 + 0.4 * rng.random(), 0.05 + 0.4 * rng.random(), 0.4 + 1.2 * rng.random(),
                          0.3 * rng.random(), *(0.8 * (rng.random(3) - 0.5))])
            sl = oracle.brdf_all_ms(p, lp, bounces) * (1 + 0.01 * rng.standard_normal(256))
            q = (p * (1 + 0.15 * rng.standard_normal(7))).astype(np.float32)
            q[:4] = np.abs(q[:4]) + 1e-3
            lum.append(sl.astype(np.float32))
            init.append(q)
        lum, init = np.asarray(lum), np.asarray(init)
        out, rmse, st = gpu_ctx.lsq_fit_batch(lp, lum, init, svf.options(multi_scattering=bounces))
        ref = np.array([oracle.lsq_fit_ms(lum[t], lp, init[t], bounces)[1] for t in range(T)])
        ratio = rmse / ref
        if bounces == 1:
            assert np.mean(ratio <= 1.01) >= 0.75 and ratio.max() <= 1.5, (bounces, ratio)
        else:
            assert np.median(ratio) <= 1.01 and np.mean(ratio <= 1.01) >= 0.6 and ratio.max() <= 2.5, (bounces, ratio)
        init_rmse = gpu_ctx.lsq_fit_batch(lp, lum, init, svf.options(max_iterations=0, multi_scattering=bounces))[1]
        assert (rmse <= init_rmse).all()


def test_fit_round_trip_ring81(gpu_ctx):
    """Render maps with svf_render_btf_ms (256 walks, seed 0: the fit's model) and
    fit their luminance with SVF_LSQ_MULTI_SCATTERING from a perturbed start on
    ring-81: the fit ends well below where it started."""
    lp = svf.directions_ring81()
    rng = np.random.default_rng(9)
    T = 4
    sigma = (0.1 + 0.3 * rng.random((T, 2))).astype(np.float32)
    ks = (0.5 + rng.random(T)).astype(np.float32)
    kd = (0.2 * rng.random(T)).astype(np.float32)
    quat = np.tile(np.array([0, 0, 0, 1], np.float32), (T, 1))
    rgb = gpu_ctx.render_btf_ms(lp, np.repeat(kd[:, None], 3, 1), np.repeat(ks[:, None], 3, 1), sigma, quat, 1)
    lum = rgb[:, :, 0].copy()   # grey albedos: every channel is the luminance
    truth = np.stack([sigma[:, 0], sigma[:, 1], ks, kd, np.zeros(T), np.zeros(T), np.zeros(T)], 1).astype(np.float32)
    init = (truth * (1 + 0.2 * rng.standard_normal((T, 7)))).astype(np.float32)
    init[:, :4] = np.abs(init[:, :4]) + 1e-3
    init[:, 4:] = 0.05 * rng.standard_normal((T, 3))
    o0 = svf.options(max_iterations=0, multi_scattering=1)
    r0 = gpu_ctx.lsq_fit_batch(lp, lum, init, o0)[1]
    out, rmse, st = gpu_ctx.lsq_fit_batch(lp, lum, init, svf.options(multi_scattering=1))
    assert (rmse <= 0.5 * r0).all(), (rmse, r0)
    # the truth is a zero of this model (the render is the fit's model)
    rt = gpu_ctx.lsq_fit_batch(lp, lum, truth, o0)[1]
    assert (rt <= 1e-4 * np.sqrt(np.mean(lum.astype(np.float64) ** 2, 1))).all(), rt


@pytest.mark.parametrize("kw", [dict(diffuse=False), dict(fit_direction=False), dict(fit_top=True),
                                dict(downsample=41)])
def test_invalid_option_combinations(gpu_ctx, kw):
    lp = svf.directions_ring81()
    lum = np.zeros((1, 81 * 81), np.float32)
    init = np.array([[0.2, 0.2, 1.0, 0.1, 0, 0, 0]], np.float32)
    with pytest.raises(svf.SvfError) as e:
        gpu_ctx.lsq_fit_batch(lp, lum, init, svf.options(multi_scattering=2, **kw))
    assert e.value.status == svf.SVF_EINVAL
