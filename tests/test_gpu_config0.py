"""The plain-LM workload as the reference runs it: 64x64 synthetic texels, 81x81
ring directions, RGB FP32, LM capped at 100 iterations, default initial guess,
against the reference's own CPU fitter on 256 of the texels
(tests/golden/ref_config0.npz, from tests/golden/make_config0_golden.py; the
reference needed at most 46 iterations there, so the cap does not bind).

* The default initial guess is the reference's (to 1e-3 on sigma, specular,
  diffuse), texel by texel.
* Started from the reference's own final parameters, the GPU LM ends within
  1.01x of the reference's RMSE on every texel (it accepts only steps that
  lower the residual, and evaluates the residual as the reference does).
* From the default initial guess LM is chaotic (one float ulp in the start moves
  the reference's own RMSE by more than 1% on some texels, see
  test_oracle_golden.py), so the final RMSEs are compared as a distribution:
  mean <= 1.01x the reference's, median ratio <= 1.001, at least 80% of the
  texels within 1.01x; the assertion messages print the whole distribution.
* The workload in full: all 4096 texels against the reference's fits of every
  texel (tests/golden/ref_config0_full.npz, `make_config0_golden.py --full`,
  bit-identical to the subset fixture on its 256 texels): from the reference's
  final parameters every texel within 1.01x, and from the default initial guess
  median ratio <= 1.001 with at least 85 % of the texels within 1.01x.  (A mean
  bar is left out here: over 4096 chaotic fits a single texel that lands in a
  far worse minimum on either side moves the mean by several percent.)
"""
import os

import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def cfg0():
    return np.load(os.path.join(HERE, "golden", "ref_config0.npz"))


@pytest.fixture(scope="module")
def cfg0_full():
    return np.load(os.path.join(HERE, "golden", "ref_config0_full.npz"))


@pytest.fixture(scope="module")
def fitted(gpu_ctx, oracle_lib, golden, cfg0):
    """All 64x64 texels, generated by the same CPU generator as the reference's
    inputs (bit-identical samples), fitted in one call."""
    m = golden["mesh"]
    lay = svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])
    side, seed, mix = int(cfg0["side"]), int(cfg0["seed"]), int(cfg0["mix"])
    T = side * side
    samples = np.stack([oracle_lib.synth_render(seed, t, oracle_lib.synth_truth(seed, mix, t), lay.lights_parabolic)
                        for t in range(T)])
    maps, rs = gpu_ctx.fit_texels(lay, samples, side, side, opts=svf.options(max_iterations=100))
    return lay, samples, maps, rs


def _distribution(ratio):
    return (f"mean {ratio.mean():.4f} median {np.median(ratio):.5f} within 1.01x {np.mean(ratio <= 1.01):.3f} "
            f"better by >1% {np.mean(ratio < 0.99):.3f} p99 {np.quantile(ratio, 0.99):.3f} max {ratio.max():.3f}")


def test_config0_default_init_is_the_references(fitted, cfg0):
    _, _, maps, rs = fitted
    assert rs.texels == 4096 and rs.failed_texels == 0
    idx = cfg0["idx"]
    np.testing.assert_allclose(maps["init"][idx][:, :4], cfg0["init"][:, :4], rtol=1e-3, atol=1e-5)


def test_config0_from_reference_optimum_per_texel(gpu_ctx, fitted, cfg0):
    lay, samples, _, _ = fitted
    idx = cfg0["idx"]
    sub = np.ascontiguousarray(samples[idx])
    maps, rs = gpu_ctx.fit_texels(lay, sub, len(idx), 1, opts=svf.options(max_iterations=100),
                                  init=np.ascontiguousarray(cfg0["fit"], np.float32), want=("rmse",))
    ratio = maps["rmse"].astype(np.float64) / cfg0["rmse"]
    assert np.all(ratio <= 1.01), _distribution(ratio)


def test_config0_from_default_init_distribution(fitted, cfg0):
    _, _, maps, _ = fitted
    idx = cfg0["idx"]
    gpu = maps["rmse"][idx].astype(np.float64)
    ratio = gpu / cfg0["rmse"]
    msg = _distribution(ratio)
    print("config 0, GPU / reference RMSE per texel:", msg)
    assert gpu.mean() <= 1.01 * cfg0["rmse"].mean(), msg
    assert np.median(ratio) <= 1.001 and np.mean(ratio <= 1.01) >= 0.80, msg


def test_config0_all_texels_from_reference_optimum(gpu_ctx, fitted, cfg0_full):
    lay, samples, _, _ = fitted
    side = int(cfg0_full["side"])
    maps, rs = gpu_ctx.fit_texels(lay, samples, side, side, opts=svf.options(max_iterations=100),
                                  init=np.ascontiguousarray(cfg0_full["fit"], np.float32), want=("rmse",))
    assert rs.texels == side * side
    ratio = maps["rmse"].astype(np.float64) / np.maximum(cfg0_full["rmse"].astype(np.float64), 1e-30)
    assert np.all(ratio <= 1.01), _distribution(ratio)


def test_config0_all_texels_from_default_init_distribution(fitted, cfg0_full):
    _, _, maps, _ = fitted
    ratio = maps["rmse"].astype(np.float64) / np.maximum(cfg0_full["rmse"].astype(np.float64), 1e-30)
    msg = _distribution(ratio)
    print("config 0 in full (4096 texels), GPU / reference RMSE per texel:", msg)
    assert len(ratio) == 4096
    assert np.median(ratio) <= 1.001 and np.mean(ratio <= 1.01) >= 0.85, msg
