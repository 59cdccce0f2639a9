"""The LM kernel's bounded slab wait, made to run out on purpose.

Each texel's luminance slab reaches shared memory by one bulk copy that
completes an mbarrier; the control warp waits for it with a bounded number of
polls.  The library's fault injection (SVF_FAULT_SKIP_SLAB_COPY, read from the
environment at each launch) leaves one texel's copy unissued, so nothing ever
completes that barrier and the wait runs out: the call must return
SVF_ETIMEOUT, the texel's status must carry SVF_TEXEL_TIMEOUT, every other texel
must still be fitted exactly as without the fault, and the context must stay
usable.  No GPU fault is involved: the wait is on a barrier that nothing sets,
bounded by SVF_FAULT_WAIT_SPINS polls.
"""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

pytestmark = pytest.mark.gpu


def _inputs(oracle_lib, golden):
    p = golden["pipeline"]
    lp = golden["mesh"]["lights_parabolic"]
    lum = []
    for x in range(8):
        t = oracle_lib.synth_truth(int(p["seed"]), int(p["mix"]), x)
        l, _ = oracle_lib.lum_slice(oracle_lib.synth_render(int(p["seed"]), x, t, lp))
        lum.append(l)
    return lp, np.stack(lum), p["init"].astype(np.float32)


def test_expired_slab_wait_reports_timeout(gpu_ctx, oracle_lib, golden, monkeypatch):
    lp, lum, init = _inputs(oracle_lib, golden)
    T = lum.shape[0]
    out_ref, rmse_ref, stats_ref = gpu_ctx.lsq_fit_batch(lp, lum, init)

    skip = 3
    monkeypatch.setenv("SVF_FAULT_SKIP_SLAB_COPY", str(skip))
    monkeypatch.setenv("SVF_FAULT_WAIT_SPINS", "4096")
    out = np.full((T, 7), np.nan, np.float32)
    rmse = np.full(T, np.nan, np.float32)
    stats = np.zeros(T, svf.STATS_DTYPE)
    with pytest.raises(svf.SvfError) as e:
        gpu_ctx.lsq_fit_batch(lp, lum, init, out=out, rmse=rmse, stats=stats)
    assert e.value.status == svf.SVF_ETIMEOUT, e.value
    assert stats["status"][skip] & svf.SVF_TEXEL_TIMEOUT
    others = np.arange(T) != skip
    assert np.array_equal(out[others], out_ref[others])
    assert np.array_equal(rmse[others], rmse_ref[others])
    assert not np.any(stats["status"][others] & svf.SVF_TEXEL_TIMEOUT)

    # the context is still usable, and without the fault the fit is the same again
    monkeypatch.delenv("SVF_FAULT_SKIP_SLAB_COPY")
    monkeypatch.delenv("SVF_FAULT_WAIT_SPINS")
    out2, rmse2, _ = gpu_ctx.lsq_fit_batch(lp, lum, init)
    assert np.array_equal(out2, out_ref) and np.array_equal(rmse2, rmse_ref)
