"""The drop-in seam, compiled and run: TempestRenderer's own SVBRDFFitPipeline
(svbrdf-fitting-pipeline.cc, cache + fit, fit():684 calling LeastSquaresFitSGGX)
linked with oracle/svf_shim.cc -- the LeastSquaresFitSGGX replacement that
INTEGRATION.md shows a maintainer adding, with the reference's signature
(svbrdf-fitting.hh:126-127) and the fit done by libsvf.so's svf_lsq_fit_sggx --
in place of its CPU fitter (oracle/_ref/libtempest_ref_svf.so, oracle/Makefile).

On the golden texels (loaded by the reference's LoadBTF), the reference pipeline
running through the shim gives:
* the reference's own default initial guess (the reference code computes it);
* the GPU's fit of that guess, bit for bit what svf_lsq_fit_sggx returns for it
  called directly;
* the output maps the reference assembles from that fit (pipeline.cc:692-697),
  equal to the maps svf_fit_texels writes from the same initial parameters
  (SVF_INIT_GIVEN) up to float rounding (its quaternion uses the GPU's sincosf; the
  colours its average chromaticity, equal to the reference's to 1e-5).
"""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def shim_fits(oracle_lib, golden):
    if not oracle_lib.ref_svf_available():
        pytest.fail("oracle/_ref/libtempest_ref_svf.so is not built (oracle/Makefile target shim)")
    p = golden["pipeline"]
    lp = golden["mesh"]["lights_parabolic"]
    tp = golden["angles"]
    rgb = np.stack([oracle_lib.synth_render(int(p["seed"]), x, oracle_lib.synth_truth(int(p["seed"]), int(p["mix"]), x),
                                            lp) for x in range(8)])
    btf = oracle_lib.RefBTF.from_texels(tp, rgb, lib=oracle_lib.ref_svf())
    fits = [btf.fit_texel(x) for x in range(8)]
    lums = [btf.lum_slice(x) for x in range(8)]
    return rgb, fits, lums


def test_shim_pipeline_uses_reference_guess_and_gpu_fit(gpu_ctx, golden, shim_fits):
    _, fits, lums = shim_fits
    p = golden["pipeline"]
    lp = golden["mesh"]["lights_parabolic"]
    for x, (r, (lum, _)) in enumerate(zip(fits, lums)):
        # the pipeline's default initial guess is the reference's (the golden run's)
        assert np.array_equal(r["init"], p["init"][x]), x
        # its fit is svf_lsq_fit_sggx's for that guess, bit for bit
        out, rmse, st = gpu_ctx.lsq_fit_sggx(lp, lum, r["init"])
        assert np.array_equal(r["fit"], out), (x, r["fit"], out)
        assert np.float32(r["rmse"]) == np.float32(rmse)
        assert r["iterations"] == st.iterations and r["effective"] == st.effective


def test_shim_pipeline_maps_equal_gpu_maps(gpu_ctx, golden, shim_fits):
    rgb, fits, _ = shim_fits
    m = golden["mesh"]
    lay = svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])
    init = np.stack([r["init"] for r in fits]).astype(np.float32)
    maps, rs = gpu_ctx.fit_texels(lay, np.ascontiguousarray(rgb), 8, 1, init=init)
    assert rs.failed_texels == 0
    for x, r in enumerate(fits):
        ref = r["maps"]   # sigma xy, quaternion xyzw, diffuse rgb, specular rgb
        np.testing.assert_array_equal(maps["params"][x], r["fit"])
        np.testing.assert_array_equal(maps["sigma"][x], ref[0:2])
        np.testing.assert_allclose(maps["basis"][x], ref[2:6], rtol=0, atol=2e-6)
        np.testing.assert_allclose(maps["diffuse"][x], ref[6:9], rtol=2e-5, atol=1e-8)
        np.testing.assert_allclose(maps["specular"][x], ref[9:12], rtol=2e-5, atol=1e-8)


@pytest.mark.parametrize("case", ["nodir", "specular", "top", "down41", "ms1"])
def test_shim_pipeline_with_options(gpu_ctx, golden, oracle_lib, case):
    """The reference pipeline through the shim with LeastSquaresFitOptions beyond the
    default -- direction fitting disabled, the specular-only fit, LSF_OPTION_FIT_TOP,
    DownSampleLightView 41, MultiScatteringBounceCount 1 (svbrdffit -m) -- gives
    svf_lsq_fit_sggx's fit of the same options, bit for bit."""
    if not oracle_lib.ref_svf_available():
        pytest.fail("oracle/_ref/libtempest_ref_svf.so is not built (oracle/Makefile target shim)")
    O = oracle_lib
    flags, down, bounces = {"nodir": (O.LSF_OPTON_DIFFUSE | O.LSF_OPTION_DISABLE_DIRECTION_FITTING, None, None),
                            "specular": (0, None, None),
                            "top": (O.LSF_OPTON_DIFFUSE | O.LSF_OPTION_FIT_TOP, None, None),
                            "down41": (O.LSF_OPTON_DIFFUSE, 41, None),
                            "ms1": (O.LSF_OPTON_DIFFUSE, None, 1)}[case]
    p = golden["pipeline"]
    lp = golden["mesh"]["lights_parabolic"]
    x = 3
    rgb = O.synth_render(int(p["seed"]), x, O.synth_truth(int(p["seed"]), int(p["mix"]), x), lp)[None]
    btf = O.RefBTF.from_texels(golden["angles"], rgb, lib=O.ref_svf())
    r = btf.fit_texel_opts(0, flags=flags, downsample=0xFFFFFFFF if down is None else down,
                           bounces=0xFFFFFFFF if bounces is None else bounces)
    lum, _ = btf.lum_slice(0)
    opts = svf.options(diffuse=bool(flags & O.LSF_OPTON_DIFFUSE),
                       fit_direction=not (flags & O.LSF_OPTION_DISABLE_DIRECTION_FITTING),
                       fit_top=bool(flags & O.LSF_OPTION_FIT_TOP), downsample=down or 0, multi_scattering=bounces)
    if bounces is not None:
        opts.flags &= ~svf.SVF_LSQ_STEP_PER_PARAMETER
    out, rmse, st = gpu_ctx.lsq_fit_sggx(lp, lum, r["init"], opts)
    assert np.array_equal(r["fit"], out), (case, r["fit"], out)
    assert np.float32(r["rmse"]) == np.float32(rmse)
