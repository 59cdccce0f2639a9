"""svf_lsq_fit_batch_noalloc: the fit for callers that must not allocate GPU
memory (an engine that owns every device allocation through its own pool, a
frame loop that must not stall on cudaMalloc).  It works in the library's static
device scratch array instead of allocating.

Called through the C ABI with device buffers, it must give exactly what the
allocating entry point svf_lsq_fit_batch gives on the same inputs, on two calls
in a row (the second call runs in scratch the first one left behind): for the
golden texels, for the largest batch the scratch holds at 81 directions (79
texels, the slabs filling all but 5416 of its 524288 floats) and for a small
layout (16 Fibonacci directions, other padding and table sizes).  The file's
name makes pytest collect it last.
"""
import ctypes as C

import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu


def _golden_inputs(oracle_lib, golden):
    p = golden["pipeline"]
    lp = golden["mesh"]["lights_parabolic"]
    lum = []
    for x in range(8):
        t = oracle_lib.synth_truth(int(p["seed"]), int(p["mix"]), x)
        l, _ = oracle_lib.lum_slice(oracle_lib.synth_render(int(p["seed"]), x, t, lp))
        lum.append(l)
    return lp, np.stack(lum), p["init"].astype(np.float32)


def _synth_inputs(oracle_lib, lp, T, seed):
    """T seeded texels of the uneven mix, started from their ground truth moved
    by a few percent (a start every texel converges from)."""
    rng = np.random.default_rng(seed)
    lum, init = [], []
    for x in range(T):
        t = oracle_lib.synth_truth(seed, 1, x)
        l, _ = oracle_lib.lum_slice(oracle_lib.synth_render(seed, x, t, lp))
        lum.append(l)
        p = oracle_lib.truth_lum_params(t).astype(np.float64)
        p[:4] *= 1.0 + 0.05 * rng.standard_normal(4)
        p[:4] = np.maximum(p[:4], 1e-3)
        p[4:] += 0.05 * rng.standard_normal(3)
        init.append(p)
    return np.stack(lum).astype(np.float32), np.stack(init).astype(np.float32)


def _run_no_alloc_twice(gpu_ctx, lp, lum, init):
    import torch

    T = lum.shape[0]
    out_ref, rmse_ref, stats_ref = gpu_ctx.lsq_fit_batch(lp, lum, init)
    assert np.all(np.isfinite(rmse_ref))

    lib = svf.load()
    dev = torch.device("cuda", 0)
    lp_d = torch.from_numpy(np.ascontiguousarray(lp, np.float32)).to(dev)
    lum_d = torch.from_numpy(lum).to(dev)            # unpadded rows: stride L*L
    init_d = torch.from_numpy(init).to(dev)
    opts = svf.options()
    for call in range(2):
        out_d = torch.full((T, 7), float("nan"), dtype=torch.float32, device=dev)
        rmse_d = torch.full((T,), float("nan"), dtype=torch.float32, device=dev)
        stats_d = torch.zeros((T, 5), dtype=torch.int32, device=dev)
        st = lib.svf_lsq_fit_batch_noalloc(lp_d.data_ptr(), lp.shape[0], lum_d.data_ptr(), lum.shape[1], T,
                                           C.byref(opts), init_d.data_ptr(), out_d.data_ptr(), rmse_d.data_ptr(),
                                           stats_d.data_ptr(), None)
        assert st == svf.SVF_OK, lib.svf_last_error()
        torch.cuda.synchronize()
        assert np.array_equal(out_d.cpu().numpy(), out_ref), call
        assert np.array_equal(rmse_d.cpu().numpy(), rmse_ref), call
        assert np.array_equal(stats_d.cpu().numpy().view(np.uint32)[:, 0], stats_ref["iterations"]), call


def test_no_alloc_matches_batch_on_two_calls(gpu_ctx, oracle_lib, golden):
    lp, lum, init = _golden_inputs(oracle_lib, golden)
    _run_no_alloc_twice(gpu_ctx, lp, lum, init)


def test_no_alloc_largest_batch_at_81_directions(gpu_ctx, oracle_lib, golden):
    lp = golden["mesh"]["lights_parabolic"]
    T = svf.SVF_NOALLOC_MAX_SLAB_FLOATS // 6568   # 79: the most the scratch holds at L = 81
    assert T == 79
    lum, init = _synth_inputs(oracle_lib, lp, T, 41)
    _run_no_alloc_twice(gpu_ctx, lp, lum, init)


def test_no_alloc_small_layout(gpu_ctx, oracle_lib):
    lp = svf.directions_fibonacci(16)
    lum, init = _synth_inputs(oracle_lib, lp, 24, 43)
    _run_no_alloc_twice(gpu_ctx, lp, lum, init)


def test_no_alloc_rejects_too_many_texels_and_non_device_buffers(oracle_lib, golden):
    import torch

    lib = svf.load()
    lp = golden["mesh"]["lights_parabolic"]
    dev = torch.device("cuda", 0)
    lp_d = torch.from_numpy(lp).to(dev)
    T = 80   # 80 * 6568 floats > SVF_NOALLOC_MAX_SLAB_FLOATS
    lum_d = torch.zeros((T, 6561), dtype=torch.float32, device=dev)
    init_d = torch.zeros((T, 7), dtype=torch.float32, device=dev)
    out_d = torch.zeros((T, 7), dtype=torch.float32, device=dev)
    rmse_d = torch.zeros(T, dtype=torch.float32, device=dev)
    opts = svf.options()
    st = lib.svf_lsq_fit_batch_noalloc(lp_d.data_ptr(), 81, lum_d.data_ptr(), 6561, T, C.byref(opts),
                                       init_d.data_ptr(), out_d.data_ptr(), rmse_d.data_ptr(), None, None)
    assert st == svf.SVF_EINVAL and b"SVF_NOALLOC_MAX_SLAB_FLOATS" in lib.svf_last_error()
    # pageable and pinned host memory are rejected before any launch
    host_lum = np.zeros((4, 6561), np.float32)
    st = lib.svf_lsq_fit_batch_noalloc(lp_d.data_ptr(), 81, host_lum.ctypes.data, 6561, 4, C.byref(opts),
                                       init_d.data_ptr(), out_d.data_ptr(), rmse_d.data_ptr(), None, None)
    assert st == svf.SVF_EINVAL and b"device memory of the current device" in lib.svf_last_error()
    pinned_out = torch.zeros((4, 7), dtype=torch.float32).pin_memory()
    st = lib.svf_lsq_fit_batch_noalloc(lp_d.data_ptr(), 81, lum_d.data_ptr(), 6561, 4, C.byref(opts),
                                       init_d.data_ptr(), pinned_out.data_ptr(), rmse_d.data_ptr(), None, None)
    assert st == svf.SVF_EINVAL and b"device memory of the current device" in lib.svf_last_error()
