"""CUDA-graph replay of a repeated svf_fit_texels call: the second identical
call (device-resident samples, device or pinned outputs) is recorded into a
graph and launched, later ones replay it, and every call gives the same maps as
the first, directly launched one.  A call whose outputs are pageable host
memory is never recorded; changing an output buffer starts over."""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu


def test_repeated_call_is_recorded_then_replayed(oracle_lib, golden):
    import torch

    m = golden["mesh"]
    lay = svf.Layout(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])
    lp = lay.lights_parabolic
    T = 96
    rgb = np.stack([oracle_lib.synth_render(12, x, oracle_lib.synth_truth(12, 1, x), lp) for x in range(T)])
    samples = torch.from_numpy(rgb).cuda()
    shapes = {"sigma": (T, 2), "basis": (T, 4), "rmse": (T,), "params": (T, 7), "init": (T, 7)}
    want = tuple(shapes)
    dev = {k: torch.zeros(s, dtype=torch.float32, device="cuda") for k, s in shapes.items()}
    with svf.Context(0) as ctx:
        modes, results = [], []
        for _ in range(4):
            for v in dev.values():
                v.zero_()
            _, rs = ctx.fit_texels(lay, samples, T, 1, want=want, out=dev)
            torch.cuda.synchronize()
            modes.append(rs.graph)
            assert rs.failed_texels == 0 and rs.texels == T and rs.ms_total > 0
            results.append({k: v.cpu().numpy().copy() for k, v in dev.items()})
        assert modes == [0, 1, 2, 2], modes
        for r in results[1:]:
            for k in shapes:
                np.testing.assert_array_equal(r[k], results[0][k], err_msg=k)
        # another output buffer: a new call, launched directly
        other = dict(dev, rmse=torch.zeros(T, dtype=torch.float32, device="cuda"))
        _, rs = ctx.fit_texels(lay, samples, T, 1, want=want, out=other)
        assert rs.graph == 0
        np.testing.assert_array_equal(other["rmse"].cpu().numpy(), results[0]["rmse"])
        # pageable host outputs are never recorded
        host_modes = [ctx.fit_texels(lay, samples, T, 1, want=("rmse",))[1].graph for _ in range(3)]
        assert host_modes == [0, 0, 0]
