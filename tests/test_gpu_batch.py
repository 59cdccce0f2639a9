"""Several BTFs of uneven sizes and two direction layouts in one call
(svf_fit_btfs): every texel's initial guess, fit and maps are those of fitting
its BTF alone with svf_fit_texels -- the pieces share LM launches, but a texel's
arithmetic does not depend on which slot, segment or launch it lands in.

A fresh context keeps both calls on the same untuned LM configuration (256
threads), so the comparison is exact."""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu


def _rgb(oracle, lp, n, seed):
    return np.stack([oracle.synth_render(seed, x, oracle.synth_truth(seed, 1, x), lp) for x in range(n)])


def test_heterogeneous_batch_matches_single_fits(oracle_lib, golden):
    import torch

    m = golden["mesh"]
    ring = svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])
    lp151 = svf.directions_fibonacci(151)
    fib = svf.Layout(lp151, *svf.triangulate(lp151))
    rgb_a = _rgb(oracle_lib, ring.lights_parabolic, 24 * 8, 5)
    rgb_b = _rgb(oracle_lib, fib.lights_parabolic, 9 * 3, 6)
    rgb_c = _rgb(oracle_lib, ring.lights_parabolic, 5 * 7, 7)
    rgb_d = _rgb(oracle_lib, fib.lights_parabolic, 16 * 2, 8)
    init_c = np.tile(np.array([0.3, 0.2, 0.5, 0.2, 0.1, -0.2, 0.3], np.float32), (35, 1))
    btfs = [
        dict(layout=ring, samples=rgb_a, width=24, height=8),
        dict(layout=fib, samples=torch.from_numpy(rgb_b.astype(np.float16)).cuda(), width=9, height=3,
             sample_type=svf.SVF_SAMPLES_F16),
        dict(layout=ring, samples=rgb_c, width=5, height=7, init=init_c),
        dict(layout=fib, samples=rgb_d, width=16, height=2),
    ]
    want = ("diffuse", "specular", "sigma", "basis", "rmse", "params", "init", "stats")
    with svf.Context(0) as ctx:
        maps, runs, total = ctx.fit_btfs(btfs, want=want)
        assert total.texels == sum(b["width"] * b["height"] for b in btfs) and total.failed_texels == 0
        for b, mp, rs in zip(btfs, maps, runs):
            T = b["width"] * b["height"]
            assert rs.texels == T
            alone, rs1 = ctx.fit_texels(b["layout"], b["samples"], b["width"], b["height"],
                                        sample_type=b.get("sample_type", svf.SVF_SAMPLES_F32), init=b.get("init"),
                                        want=want)
            for k in ("params", "rmse", "init", "diffuse", "specular", "sigma", "basis"):
                np.testing.assert_array_equal(mp[k], alone[k], err_msg=k)
            np.testing.assert_array_equal(mp["stats"]["iterations"], alone["stats"]["iterations"])
            assert rs.jacobians == rs1.jacobians and rs.residuals == rs1.residuals


def test_batch_argument_checks(gpu_ctx, golden):
    m = golden["mesh"]
    ring = svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])
    rgb = np.zeros((4, 81 * 81, 3), np.float32)
    o1 = svf.options(max_iterations=10)
    with pytest.raises(svf.SvfError):   # GIVEN init without parameters is caught in the wrapper's options
        lib = svf.load()
        views = (svf.BtfView * 2)()
        fos = (svf.FitOptions * 2)()
        ms = (svf.Maps * 2)()
        for i in range(2):
            views[i].samples = rgb.ctypes.data
            views[i].sample_type = svf.SVF_SAMPLES_F32
            views[i].width, views[i].height = 2, 2
            views[i].layout = svf.C.pointer(ring.desc)
            fos[i].lsq = o1
        fos[1].lsq.max_iterations = 20   # different lsq options in one call
        svf._check(lib.svf_fit_btfs(gpu_ctx.handle, views, 2, fos, ms, None, None))
    assert "same for every BTF" in svf.load().svf_last_error().decode()
