"""The luminance pass's two ways of reading samples (svf_kernels.cu): FP32
samples straight into registers, FP16 samples staged through shared memory by
16-byte cp.async copies with the ragged first and last bytes loaded one by one,
and the feature variant that keeps the slab in shared memory in bin order.

FP16 samples and the same values widened to FP32 give the same luminance, BF16
split and average chromaticity, so every output of the fit is bit-identical
between the two sample types -- at each of the eight 2-byte alignments a texel
range of FP16 samples can start at (a texel is 39366 bytes at 81 directions,
6 mod 16), since a texel's fit does not depend on the launch it runs in.  The
learned guess's features agree the same way."""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu

WANT = ("diffuse", "specular", "sigma", "basis", "rmse", "params", "init", "stats")


def _layout(golden):
    m = golden["mesh"]
    return svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])


def test_fp16_staging_matches_fp32_at_every_alignment(gpu_ctx, golden):
    import torch

    lay = _layout(golden)
    T, n = 72, 64
    s32 = torch.empty((T, 81 * 81, 3), dtype=torch.float32, device="cuda")
    gpu_ctx.synth_btf(4242, 1, lay.lights_parabolic, 0, T, s32)
    s16 = s32.half()
    wide = s16.float()   # the FP16 values in FP32
    ref, _ = gpu_ctx.fit_texels(lay, wide, T, 1, want=WANT)
    for k in range(8):   # byte offsets 6k mod 16: 0, 6, 12, 2, 8, 14, 4, 10
        got, rs = gpu_ctx.fit_texels(lay, s16[k:k + n], n, 1, sample_type=svf.SVF_SAMPLES_F16, want=WANT)
        assert rs.failed_texels == 0
        for key in WANT:
            np.testing.assert_array_equal(got[key], ref[key][k:k + n], err_msg=f"{key} at offset {k}")
    # host FP16 samples (staged into the library's pinned buffers) take the same path
    got, _ = gpu_ctx.fit_texels(lay, s16[3:3 + n].cpu().numpy(), n, 1, sample_type=svf.SVF_SAMPLES_F16, want=WANT)
    for key in WANT:
        np.testing.assert_array_equal(got[key], ref[key][3:3 + n], err_msg=key)


def test_feature_pass_matches_across_sample_types(gpu_ctx, golden):
    import torch

    from test_gpu_mlp import _blob, _random_model

    lay = _layout(golden)
    lp = lay.lights_parabolic
    m = svf.Mlp.load(gpu_ctx, _blob(lp, *_random_model(lp, 5, scale=0.05)))
    T, n = 40, 32
    s32 = torch.empty((T, 81 * 81, 3), dtype=torch.float32, device="cuda")
    gpu_ctx.synth_btf(99, 1, lp, 0, T, s32)
    s16 = s32.half()
    wide = s16.float()
    p_ref, f_ref = m.predict(wide, T, features=True)
    for k in (0, 1, 5):
        p, f = m.predict(s16[k:k + n], n, sample_type=svf.SVF_SAMPLES_F16, features=True)
        np.testing.assert_array_equal(f, f_ref[k:k + n])
        np.testing.assert_array_equal(p, p_ref[k:k + n])
    # and the fit from the learned guess starts at the prediction
    got, _ = gpu_ctx.fit_texels(lay, s16[1:1 + n], n, 1, sample_type=svf.SVF_SAMPLES_F16, mlp=m,
                                want=("init", "rmse"))
    np.testing.assert_array_equal(got["init"], p_ref[1:1 + n])
    m.close()
