"""The fit on the 151-direction Fibonacci hemisphere (22801 direction pairs per
texel, 91 KB luminance slabs), in FP32 and FP16 sample storage: the BRDF and
residual evaluation against the FP64 oracle, LM from a good start against the
oracle LM, and the default initial guess against the oracle's, with the
library's own triangulation of the directions as the interpolation mesh.

Tolerances are those of test_gpu_lsq.py and test_gpu_pipeline.py."""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu

L151 = 151
SEED = 57


@pytest.fixture(scope="module")
def fib():
    lp = svf.directions_fibonacci(L151)
    tri, edges, ang = svf.triangulate(lp)
    return lp, tri, edges, ang


def _texels(oracle, lp, n, seed=SEED):
    rgb, lum, truth = [], [], []
    for x in range(n):
        t = oracle.synth_truth(seed, 1, x)
        c = oracle.synth_render(seed, x, t, lp)
        rgb.append(c)
        lum.append(oracle.lum_slice(c)[0])
        truth.append(oracle.truth_lum_params(t))
    return np.stack(rgb), np.stack(lum), np.stack(truth)


def test_brdf_and_residual_at_151_directions(gpu_ctx, oracle_lib, fib):
    lp = fib[0]
    _, lum, truth = _texels(oracle_lib, lp, 3)
    for x in range(3):
        p = truth[x].astype(np.float64)
        f32, f64 = oracle_lib.brdf_all(p, lp)
        # zero-iteration fit of the FP64 model values: its RMSE is the model error
        _, rmse, st = gpu_ctx.lsq_fit_sggx(lp, f64.astype(np.float32), p.astype(np.float32),
                                           svf.options(max_iterations=0))
        assert rmse / np.sqrt(np.mean(f64 ** 2)) <= 1e-5
        expect = np.sqrt(np.mean((lum[x].astype(np.float64) - f32) ** 2))
        _, rmse, _ = gpu_ctx.lsq_fit_sggx(lp, lum[x], p.astype(np.float32), svf.options(max_iterations=0))
        np.testing.assert_allclose(rmse, expect, rtol=1e-4)


def test_lm_from_good_start_at_151_directions(gpu_ctx, oracle_lib, fib):
    from test_gpu_lsq import parity_stats

    lp = fib[0]
    T = 8
    _, lum, truth = _texels(oracle_lib, lp, T)
    rng = np.random.default_rng(3)
    init = (truth * (1 + 0.15 * rng.standard_normal(truth.shape))).astype(np.float32)
    init[:, :4] = np.abs(init[:, :4]) + 1e-3
    out, rmse, stats = gpu_ctx.lsq_fit_batch(lp, lum, init)
    assert (stats["status"] == 0).all()
    ref = np.array([oracle_lib.lsq_fit(lum[t], lp, init[t])[1] for t in range(T)])
    mean_ratio, within, worst = parity_stats(rmse, ref)
    assert mean_ratio <= 1.01 and within >= 0.75, (np.c_[rmse, ref], mean_ratio, within)


def test_default_init_and_fp16_storage_at_151_directions(gpu_ctx, oracle_lib, fib):
    from test_gpu_lsq import parity_stats

    lp, tri, edges, ang = fib
    lay = svf.Layout(lp, tri, edges, ang)
    T = 6
    rgb, lum, _ = _texels(oracle_lib, lp, T)
    maps32, rs = gpu_ctx.fit_texels(lay, rgb, T, 1, want=("init", "rmse", "params", "ndf"))
    assert rs.failed_texels == 0 and np.isfinite(maps32["rmse"]).all()
    # the default initial guess of one texel against the oracle's, on the same mesh
    mesh = oracle_lib.MeshData(lp, tri, edges, ang)
    ndf = oracle_lib.ndf_texture(mesh, lum[0])
    peak = float(np.abs(ndf).max())
    assert float(np.abs(maps32["ndf"][0] - ndf).max()) <= 1e-4 * peak
    init, _ = oracle_lib.default_init_from_ndf(ndf)
    gi = maps32["init"][0]
    np.testing.assert_allclose(gi[:4], init[:4], rtol=1e-3, atol=1e-6)
    mg, _ = oracle_lib.euler_to_matrix(gi[4:7])
    mr, _ = oracle_lib.euler_to_matrix(init[4:7])
    np.testing.assert_allclose(mg, mr, atol=1e-3)
    # FP16 storage of the same texels: the fit lands within the statistical bar of the FP32 one
    maps16, rs16 = gpu_ctx.fit_texels(lay, rgb.astype(np.float16), T, 1, sample_type=svf.SVF_SAMPLES_F16,
                                      want=("rmse",))
    assert rs16.failed_texels == 0
    mean_ratio, within, worst = parity_stats(maps16["rmse"], maps32["rmse"])
    assert mean_ratio <= 1.05 and within >= 0.5, (np.c_[maps16["rmse"], maps32["rmse"]], mean_ratio)
