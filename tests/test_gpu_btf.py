"""Factored BTF files on the GPU (svf_btf_load / svf_btf_decode / svf_fit_btf):

* every golden file decodes to what the reference's BTFFetchSpectrum returned
  (tests/golden/ref_btf.npz): bit for bit where no exponential is involved,
  within 4 ulp-scale relative error with colour model 11 or the dynamic range
  reduction (CUDA's expf against libm's);
* a larger ring-81 file with realistic plane sizes decodes bit-identically to
  the oracle restatement (pinned to the reference by test_btf_file.py), in FP32
  and FP16 output, on the device and to host memory, whole and by sub-range;
* svf_fit_btf equals svf_fit_texels on the decoded samples, and on a file
  holding the golden pipeline's texels it reproduces the reference's fits."""
import os

import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu

# colour model 11 and DRR go through expf: CUDA's differs from libm's by at most
# 2 ulp, and the YUV -> RGB combination can cancel, so the bound is relative to
# the sample's magnitude plus a small absolute floor
EXP_RTOL, EXP_ATOL = 2e-6, 1e-7


@pytest.fixture(scope="module")
def ref_btf():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_btf.npz"))


def test_golden_files_decode_like_loadbtf(gpu_ctx, ref_btf):
    for name in ref_btf["names"]:
        name = str(name)
        data = ref_btf[f"{name}/bytes"].tobytes()
        if not bool(ref_btf[f"{name}/ok"]):
            with pytest.raises(svf.SvfError):
                svf.Btf(gpu_ctx, data)
            continue
        b = svf.Btf(gpu_ctx, data)
        ref = ref_btf[f"{name}/spectra"]
        got = b.decode()
        fmt, ds, cm, drr, W, H, L = (int(v) for v in ref_btf[f"{name}/meta"])
        if cm == 0 and drr == 0:
            np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32), err_msg=name)
            np.testing.assert_array_equal(b.decode(sample_type=svf.SVF_SAMPLES_F16), ref.astype(np.float16),
                                          err_msg=name)
        else:
            np.testing.assert_allclose(got, ref, rtol=EXP_RTOL, atol=EXP_ATOL, err_msg=name)
        np.testing.assert_array_equal(b.lights_parabolic, ref_btf[f"{name}/lights_parabolic"])
        b.close()


def _ring_file(oracle, fmt, ds, ks, W, H, seed, cm=0, drr=0, scale=0.2):
    tp = oracle.ring81_angles()
    N, T = 81 * 81, W * H
    rng = np.random.default_rng(seed)
    if fmt == "DFMF":
        planes = [(rng.normal(0, scale, (N, k)), rng.normal(0, scale, (T, k))) for k in ks]
    else:
        planes = (rng.normal(0, scale, (N * 3, ks[0])), rng.normal(0, scale, (T, ks[0])))
    return planes, oracle.btf_file_bytes(tp, W, H, planes, fmt=fmt, data_size=ds, color_model=cm, drr=drr)


# (150 components: five 32-component chunks, the last one partial)
@pytest.mark.parametrize("fmt,ds,ks,drr", [("DFMF", 2, (24, 16, 40), 0), ("DFMF", 4, (33, 8, 20), 0),
                                           ("FMF1", 2, (28,), 1), ("DFMF", 8, (12, 12, 12), 0),
                                           ("DFMF", 4, (150, 40, 9), 0)])
def test_ring81_decode_matches_oracle(gpu_ctx, oracle_lib, fmt, ds, ks, drr):
    import torch

    W, H = 37, 9   # ragged against the 16-texel groups and the 128-pair blocks
    planes, data = _ring_file(oracle_lib, fmt, ds, ks, W, H, seed=len(ks) * 7 + ds, drr=drr)
    b = svf.Btf(gpu_ctx, data)
    ref = oracle_lib.btf_decode(planes, fmt, W, H, 81, ds, 0, drr)
    dev = torch.empty((W * H, 81 * 81, 3), dtype=torch.float32, device="cuda")
    b.decode(out=dev)
    got = dev.cpu().numpy()
    if drr == 0:
        np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32))
    else:
        np.testing.assert_allclose(got, ref, rtol=EXP_RTOL, atol=EXP_ATOL)
    # host output and a sub-range give the same samples
    np.testing.assert_array_equal(b.decode(first=50, count=100), got[50:150])
    h16 = b.decode(sample_type=svf.SVF_SAMPLES_F16)
    np.testing.assert_array_equal(h16, got.astype(np.float16))
    with pytest.raises(svf.SvfError):
        b.decode(first=W * H - 1, count=2)
    b.close()


def test_fit_btf_equals_fit_of_decoded_samples(gpu_ctx, oracle_lib, golden):
    """Synthetic texels written as a DFMF file (U = the samples, SxV = identity),
    fitted straight from the file: maps equal fitting the decoded samples."""
    m = golden["mesh"]
    lay = svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])
    lp = lay.lights_parabolic
    W, H = 24, 5
    rgb = np.stack([oracle_lib.synth_render(91, x, oracle_lib.synth_truth(91, 1, x), lp) for x in range(W * H)])
    # file column (H-1-y)*W + x holds texel y*W + x
    cols = np.array([(H - 1 - (t // W)) * W + t % W for t in range(W * H)])
    planes = []
    for c in range(3):
        U = rgb[:, :, c].T.astype(np.float32)                  # [N][K = T]
        S = np.zeros((W * H, W * H), np.float32)
        S[cols, np.arange(W * H)] = 1.0                        # column of texel t picks U's column t
        planes.append((U, S))
    data = oracle_lib.btf_file_bytes(golden["angles"], W, H, planes, data_size=4)
    b = svf.Btf(gpu_ctx, data)
    dec = b.decode()
    np.testing.assert_array_equal(dec, rgb)   # one product with 1.0 per sample: exact
    want = ("diffuse", "specular", "sigma", "basis", "rmse", "params", "init", "stats")
    fb, rs = b.fit(layout=lay, want=want)
    ft, _ = gpu_ctx.fit_texels(lay, dec, W, H, want=want)
    assert rs.texels == W * H and rs.failed_texels == 0
    for k in want:
        np.testing.assert_array_equal(fb[k], ft[k], err_msg=k)
    # the RGB fit takes the same route
    rgb_b, _ = b.fit(layout=lay, opts=svf.options(rgb=True), want=("params", "rmse"))
    rgb_t, _ = gpu_ctx.fit_texels(lay, dec, W, H, opts=svf.options(rgb=True), want=("params", "rmse"))
    np.testing.assert_array_equal(rgb_b["params"], rgb_t["params"])
    b.close()


def test_fit_btf_reproduces_reference_pipeline(gpu_ctx, oracle_lib, golden):
    """The golden pipeline's eight texels in a DFMF file (as the golden generator
    wrote them for the reference's LoadBTF): the fits' residuals meet the
    reference's within the pipeline test's bar."""
    from test_gpu_lsq import parity_stats

    p = golden["pipeline"]
    m = golden["mesh"]
    lp = m["lights_parabolic"]
    seed, mix = int(p["seed"]), int(p["mix"])
    rgb = np.stack([oracle_lib.synth_render(seed, x, oracle_lib.synth_truth(seed, mix, x), lp) for x in range(8)])
    planes = [(rgb[:, :, c].T.astype(np.float32), np.eye(8, dtype=np.float32)) for c in range(3)]
    data = oracle_lib.btf_file_bytes(golden["angles"], 8, 1, planes, data_size=4)
    b = svf.Btf(gpu_ctx, data)
    lay = svf.Layout(lp, m["triangles"], m["edges"], m["edge_angles"])
    maps, rs = b.fit(layout=lay, want=("rmse", "init"))
    assert rs.failed_texels == 0
    mean_ratio, within, worst = parity_stats(maps["rmse"], np.asarray(p["rmse"]))
    assert mean_ratio <= 1.01 and within >= 0.75, (mean_ratio, within, worst)
    b.close()
