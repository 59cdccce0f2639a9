"""GPU LeastSquaresFitSGGX (svf_lsq_fit_sggx / svf_lsq_fit_batch) against the
oracle and the reference's golden fits.

Tolerances:
* BRDF: the RMS of (GPU f32 - FP64 model) over all pairs, relative to the RMS
  of the FP64 values, is <= 1e-5 (observed through a zero-iteration fit, whose
  RMSE is the RMS of the model error against the slice it is given).
* Fit from a good start (the golden fits' perturbed ground truth): per texel,
  final RMSE <= 1.01 x the reference's + 1e-7.
* Fit from a rough start (ground truth moved by 15 % per parameter, 64 texels
  of the uneven mix, every one of them also fitted by the oracle): such starts
  reach the chaotic regime too, so the bar is the statistical one below.
* Fit from the reference's default initial guess: LM from that rough start is
  chaotic -- the reference itself, started one float ulp away, ends more than
  1.01x worse on 2 of the 8 golden texels (5.6x on one; see
  test_oracle_golden.py::test_reference_lm_is_sensitive_to_one_ulp).  The bar
  is therefore statistical: mean RMSE <= 1.01 x the reference's mean, at least
  3/4 of the texels within 1.01x, none worse than 1.25x.
"""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu


def _lp(golden):
    return golden["mesh"]["lights_parabolic"]


def _texel_lum(oracle, golden, x):
    p = golden["pipeline"]
    t = oracle.synth_truth(int(p["seed"]), int(p["mix"]), x)
    rgb = oracle.synth_render(int(p["seed"]), x, t, _lp(golden))
    lum, _ = oracle.lum_slice(rgb)
    return lum


def test_brdf_relative_error_vs_fp64(gpu_ctx, oracle_lib, golden):
    lp = _lp(golden)
    params = golden["lsq"]["brdf_params"]
    for p in params[:4]:
        _, f64 = oracle_lib.brdf_all(p, lp)
        lum = f64.astype(np.float32)
        out, rmse, st = gpu_ctx.lsq_fit_sggx(lp, lum, p.astype(np.float32), svf.options(max_iterations=0))
        rel = rmse / np.sqrt(np.mean(f64 ** 2))
        assert rel <= 1e-5, (p, rel)
        assert st.iterations == 0 and np.array_equal(out, p.astype(np.float32))


def test_residual_matches_oracle_at_other_parameters(gpu_ctx, oracle_lib, golden):
    lp = _lp(golden)
    lum = _texel_lum(oracle_lib, golden, 2)
    for p in golden["lsq"]["brdf_params"]:
        f32, _ = oracle_lib.brdf_all(p, lp)
        expect = np.sqrt(np.mean((lum.astype(np.float64) - f32) ** 2))
        _, rmse, _ = gpu_ctx.lsq_fit_sggx(lp, lum, p.astype(np.float32), svf.options(max_iterations=0))
        np.testing.assert_allclose(rmse, expect, rtol=1e-4)


def parity_stats(rmse, ref):
    rmse, ref = np.asarray(rmse, np.float64), np.asarray(ref, np.float64)
    within = rmse <= 1.01 * ref + 1e-7
    return float(rmse.mean() / ref.mean()), float(within.mean()), float((rmse / ref).max())


def test_fit_from_reference_default_init(gpu_ctx, oracle_lib, golden):
    p = golden["pipeline"]
    rmse = []
    for x in range(8):
        lum = _texel_lum(oracle_lib, golden, x)
        out, r, st = gpu_ctx.lsq_fit_sggx(_lp(golden), lum, p["init"][x])
        assert st.status == 0
        rmse.append(r)
    mean_ratio, within, worst = parity_stats(rmse, p["rmse"])
    assert mean_ratio <= 1.01 and within >= 0.75 and worst <= 1.25, (np.c_[rmse, p["rmse"]], mean_ratio, within)


def test_single_iteration_bound_rule(gpu_ctx, oracle_lib, golden):
    """With diffuse exactly 0 the fit must still move it: the default initial
    guess always starts there (svbrdf-fitting-pipeline.cc:659)."""
    p = golden["pipeline"]
    lum = _texel_lum(oracle_lib, golden, 0)
    out, rmse, st = gpu_ctx.lsq_fit_sggx(_lp(golden), lum, p["init"][0])
    assert p["init"][0][3] == 0.0 and out[3] > 0.1
    assert rmse < 2 * p["rmse"][0]


def test_fit_from_perturbed_truth_batch(gpu_ctx, oracle_lib, golden):
    g = golden["lsq"]
    lum = np.stack([_texel_lum(oracle_lib, golden, x) for x in range(8)])
    out, rmse, stats = gpu_ctx.lsq_fit_batch(_lp(golden), lum, g["init"].astype(np.float32))
    assert (rmse <= 1.01 * g["rmse"] + 1e-7).all(), np.c_[rmse, g["rmse"]]
    assert (stats["status"] == 0).all()


def test_batch_matches_single_and_device_pointers(gpu_ctx, oracle_lib, golden):
    import torch

    lp = _lp(golden)
    g = golden["lsq"]
    lum = np.stack([_texel_lum(oracle_lib, golden, x) for x in range(8)])
    init = g["init"].astype(np.float32)
    out_h, rmse_h, st_h = gpu_ctx.lsq_fit_batch(lp, lum, init)
    # padded stride, device buffers
    lum_d = torch.zeros((8, 6600), dtype=torch.float32, device="cuda")
    lum_d[:, :6561] = torch.from_numpy(lum).cuda()
    init_d = torch.from_numpy(init).cuda()
    out_d = torch.zeros((8, 7), dtype=torch.float32, device="cuda")
    rmse_d = torch.zeros(8, dtype=torch.float32, device="cuda")
    gpu_ctx.lsq_fit_batch(lp, lum_d, init_d, out=out_d, rmse=rmse_d, stats=np.zeros(8, svf.STATS_DTYPE))
    torch.cuda.synchronize()
    assert np.array_equal(out_d.cpu().numpy(), out_h)
    assert np.array_equal(rmse_d.cpu().numpy(), rmse_h)
    for x in (0, 5):
        o1, r1, s1 = gpu_ctx.lsq_fit_sggx(lp, lum[x], init[x])
        assert np.array_equal(o1, out_h[x]) and r1 == rmse_h[x]


def test_many_texels_against_oracle(gpu_ctx, oracle_lib, golden):
    """64 texels of the uneven parameter mix, each fitted by the GPU and by the
    oracle LM (the reference's, bit for bit) from the same rough start."""
    lp = _lp(golden)
    T = 64
    lums, inits, ref_rmse = [], [], []
    rng = np.random.default_rng(1)
    for t in range(T):
        tr = oracle_lib.synth_truth(91, 1, t)
        rgb = oracle_lib.synth_render(91, t, tr, lp)
        lum, _ = oracle_lib.lum_slice(rgb)
        truth = oracle_lib.truth_lum_params(tr)
        init = (truth * (1 + 0.15 * rng.standard_normal(7))).astype(np.float32)
        init[:4] = np.abs(init[:4]) + 1e-3
        lums.append(lum)
        inits.append(init)
    lums = np.stack(lums)
    inits = np.stack(inits)
    out, rmse, stats = gpu_ctx.lsq_fit_batch(lp, lums, inits)
    for t in range(T):
        _, r, _ = oracle_lib.lsq_fit(lums[t], lp, inits[t])
        ref_rmse.append(r)
    ref_rmse = np.array(ref_rmse)
    mean_ratio, within, worst = parity_stats(rmse, ref_rmse)
    assert mean_ratio <= 1.01 and within >= 0.75, (np.c_[rmse, ref_rmse], mean_ratio, within, worst)


def test_nonfinite_texel_is_flagged(gpu_ctx, oracle_lib, golden):
    lp = _lp(golden)
    g = golden["lsq"]
    lum = np.stack([_texel_lum(oracle_lib, golden, x) for x in range(3)])
    lum[1, 100] = np.nan
    out = np.zeros((3, 7), np.float32)
    rmse = np.zeros(3, np.float32)
    stats = np.zeros(3, svf.STATS_DTYPE)
    with pytest.raises(svf.SvfError) as e:
        gpu_ctx.lsq_fit_batch(lp, lum, g["init"][:3].astype(np.float32), out=out, rmse=rmse, stats=stats)
    assert e.value.status == svf.SVF_EPARTIAL
    assert stats["status"][1] & svf.SVF_TEXEL_NONFINITE
    assert stats["status"][0] == 0 and stats["status"][2] == 0
    assert rmse[0] <= 1.01 * g["rmse"][0] + 1e-7


def test_invalid_arguments(gpu_ctx, golden):
    lp = _lp(golden)
    lum = np.zeros(81 * 81, np.float32)
    with pytest.raises(svf.SvfError) as e:
        gpu_ctx.lsq_fit_sggx(lp, lum, np.zeros(7, np.float32), svf.options(fresnel=0.5))
    assert e.value.status == svf.SVF_EINVAL
    o = svf.options()
    o.flags |= 1 << 20   # no such option
    with pytest.raises(svf.SvfError):
        gpu_ctx.lsq_fit_sggx(lp, lum, np.zeros(7, np.float32), o)
