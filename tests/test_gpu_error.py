"""svbrdf-error-tool on the GPU (svf_error_maps): per-texel RMSE and PSNR of
fitted maps against a BTF, against the reference's own computation
(tests/golden/ref_error.npz, made by tests/golden/make_error_golden.py):
pair-wise and max-view, luminance and per channel, 2- and 3-channel scale maps,
a region offset inside the BTF.  The BRDF values differ in FP32 rounding (this
library's factored model against the reference's SGGXMicroFlakeSurfaceBRDF,
both within about 1e-5 of the FP64 value, more where a narrow lobe's peak is
large) and the reference sums squared residuals in FP32 while this library
sums in FP64, so RMSEs agree to 2e-4 relative and PSNRs to 2e-3 dB.  And the file-to-file loop: fit -> EXR maps ->
read back -> error, whose luminance RMSE is the fit's own."""
import hashlib
import os
import sys

import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))


@pytest.fixture(scope="module")
def ref_error():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_error.npz"))


def test_error_maps_match_reference(gpu_ctx, ref_error):
    import make_error_golden as G

    data, diffuse, specular, sigma, sigma3, basis = G.error_case()
    assert hashlib.sha256(data).digest() == ref_error["error/btf_sha256"].tobytes()
    b = svf.Btf(gpu_ctx, data)
    for method in (svf.SVF_ERROR_PAIRWISE, svf.SVF_ERROR_MAX_VIEW):
        for color in (0, 1):
            ref_r = ref_error[f"error/{method}/{color}/rmse"]
            ref_p = ref_error[f"error/{method}/{color}/psnr"]
            for sg in (sigma, sigma3):
                rmse, psnr = b.error_maps(diffuse, specular, sg, basis, x0=G.X0, y0=G.Y0, method=method,
                                          color=bool(color))
                rmse = rmse.reshape(ref_r.shape)
                psnr = psnr.reshape(ref_p.shape)
                np.testing.assert_allclose(rmse, ref_r, rtol=2e-4, err_msg=f"{method} {color}")
                np.testing.assert_allclose(psnr, ref_p, atol=2e-3, err_msg=f"{method} {color}")
    with pytest.raises(svf.SvfError):   # the region must lie inside the BTF
        b.error_maps(diffuse, specular, sigma, basis, x0=G.W - 1, y0=0)
    b.close()


def test_fit_to_exr_to_error_loop(gpu_ctx, oracle_lib, golden, tmp_path):
    """svbrdffit's file-to-file loop: fit a DFMF file, write the maps as EXR, read
    them back and measure them with the error tool.  With the fit's maps the
    tool's luminance RMSE is the fit's RMSE (the albedos are kd, ks times the
    average chromaticity, whose luminance is 1 up to rounding)."""
    m = golden["mesh"]
    lay = svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])
    lp = lay.lights_parabolic
    W, H = 8, 3
    rgb = np.stack([oracle_lib.synth_render(33, x, oracle_lib.synth_truth(33, 1, x), lp) for x in range(W * H)])
    cols = np.array([(H - 1 - t // W) * W + t % W for t in range(W * H)])
    planes = []
    for c in range(3):
        S = np.zeros((W * H, W * H), np.float32)
        S[cols, np.arange(W * H)] = 1.0
        planes.append((rgb[:, :, c].T.astype(np.float32), S))
    b = svf.Btf(gpu_ctx, oracle_lib.btf_file_bytes(golden["angles"], W, H, planes, data_size=4))
    maps, rs = b.fit(layout=lay, want=("diffuse", "specular", "sigma", "basis", "rmse"))
    assert rs.failed_texels == 0
    prefix = str(tmp_path / "btf")
    svf.maps_write_exr(prefix, W, H, maps)
    back = {k: svf.exr_read(f"{prefix}_{s}.exr") for k, s in (("diffuse", "albedo"), ("specular", "specular"),
                                                                ("sigma", "sggx_scale"), ("basis", "sggx_basis"),
                                                                ("rmse", "rmse"))}
    np.testing.assert_array_equal(back["rmse"].reshape(-1), maps["rmse"])
    rmse, psnr = b.error_maps(back["diffuse"], back["specular"], back["sigma"], back["basis"])
    np.testing.assert_allclose(rmse.reshape(-1), maps["rmse"], rtol=1e-4)
    assert np.all(np.isfinite(psnr))
    b.close()
