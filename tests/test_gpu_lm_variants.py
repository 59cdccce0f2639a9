"""Every LM kernel configuration (CTA size, texel slots, plain, paired-FP32 or
tensor-core J^T J pair pass) on the same checks, pinned with SVF_LM_KERNEL:

* the residual at given parameters (zero-iteration fits) equals the oracle's to
  1e-4 relative, so the pair pass evaluates the reference's BRDFEvaluator;
* from perturbed ground truth every texel ends within 1.01x of the reference's
  RMSE (tests/golden/ref_lsq.npz), so J^T J and J^T r drive LM to the optimum;
* a batch of 96 texels ends where the first (plain) configuration ends: median
  relative RMSE difference below 1e-4, at least 90% of the texels within 1e-3
  (the packed pass sums in another order and the tensor-core pass forms J^T J
  from TF32 products, so their fits are equal up to rounding, not bit for bit,
  and a rounding difference can move a narrow lobe's fit).
"""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu

# threads, slots, pair pass (0 plain, 1 paired FP32, 2 J^T J on the tensor cores)
CONFIGS = ["256,3,0", "256,2,0", "128,3,0", "128,2,0", "256,1,0", "160,2,0", "160,3,0", "256,3,1", "256,4,1",
           "128,3,1", "256,2,2", "128,3,2"]


def _lp(golden):
    return golden["mesh"]["lights_parabolic"]


def _texel_lum(oracle, seed, mix, x, lp):
    t = oracle.synth_truth(seed, mix, x)
    lum, _ = oracle.lum_slice(oracle.synth_render(seed, x, t, lp))
    return lum, oracle.truth_lum_params(t)


@pytest.fixture(scope="module")
def batch96(oracle_lib, golden):
    lp = _lp(golden)
    rng = np.random.default_rng(9)
    lum, init = [], []
    for x in range(96):
        l, t = _texel_lum(oracle_lib, 61, 1, x, lp)
        p = t.astype(np.float64) * (1 + 0.1 * rng.standard_normal(7))
        p[:4] = np.abs(p[:4]) + 1e-3
        lum.append(l)
        init.append(p)
    return np.stack(lum), np.stack(init).astype(np.float32)


@pytest.fixture(scope="module")
def plain_batch(gpu_ctx, golden, batch96):
    import os

    os.environ["SVF_LM_KERNEL"] = CONFIGS[0]
    try:
        return gpu_ctx.lsq_fit_batch(_lp(golden), *batch96)
    finally:
        del os.environ["SVF_LM_KERNEL"]


@pytest.mark.parametrize("config", CONFIGS)
def test_lm_configuration(gpu_ctx, oracle_lib, golden, batch96, plain_batch, config, monkeypatch):
    monkeypatch.setenv("SVF_LM_KERNEL", config)
    lp = _lp(golden)
    # residual at given parameters
    p = golden["pipeline"]
    lum0, _ = _texel_lum(oracle_lib, int(p["seed"]), int(p["mix"]), 2, lp)
    for q in golden["lsq"]["brdf_params"]:
        f32, _ = oracle_lib.brdf_all(q, lp)
        expect = np.sqrt(np.mean((lum0.astype(np.float64) - f32) ** 2))
        _, rmse, _ = gpu_ctx.lsq_fit_batch(lp, lum0[None], q.astype(np.float32)[None],
                                           svf.options(max_iterations=0))
        np.testing.assert_allclose(rmse[0], expect, rtol=1e-4)
    # from perturbed ground truth, against the reference
    g = golden["lsq"]
    lum8 = np.stack([_texel_lum(oracle_lib, int(p["seed"]), int(p["mix"]), x, lp)[0] for x in range(8)])
    _, rmse8, st8 = gpu_ctx.lsq_fit_batch(lp, lum8, g["init"].astype(np.float32))
    assert (rmse8 <= 1.01 * g["rmse"] + 1e-7).all(), np.c_[rmse8, g["rmse"]]
    assert (st8["status"] == 0).all()
    # a larger batch against the first configuration
    _, rmse, st = gpu_ctx.lsq_fit_batch(lp, *batch96)
    ref = plain_batch[1]
    assert (st["status"] & (svf.SVF_TEXEL_NONFINITE | svf.SVF_TEXEL_TIMEOUT) == 0).all()
    dev = np.abs(rmse.astype(np.float64) / ref - 1.0)
    assert np.median(dev) < 1e-4 and np.mean(dev <= 1e-3) >= 0.90, np.sort(dev)[-8:]
    assert rmse.mean() <= 1.01 * ref.mean()


def test_default_configuration_rule():
    """Without SVF_LM_KERNEL the configuration comes from the occupancy rule
    (svf::lm_default_choice), which ranks configurations as full B200 launches
    measured them: 160 threads x 2 slots on ring-81 slabs (three CTAs per SM),
    256 x 2 on Fibonacci-151 slabs (one CTA per SM fits two 91 KB slabs)."""
    import os

    import oracle

    assert "SVF_LM_KERNEL" not in os.environ
    for lp, want in ((svf.directions_ring81(), (160, 2)), (svf.directions_fibonacci(151), (256, 2))):
        L = lp.shape[0]
        tri, edges, angles = svf.triangulate(lp)
        layout = svf.Layout(lp, tri, edges, angles)
        rgb = np.stack([oracle.synth_render(3, t, oracle.synth_truth(3, 1, t), lp) for t in range(2)])
        with svf.Context(0) as ctx:   # (a fresh context: the configuration is chosen per layout)
            _, run = ctx.fit_texels(layout, rgb, 2, 1, want=("rmse",))
        assert (run.lm_threads, run.lm_slots) == want, (L, run.lm_threads, run.lm_slots)
