"""Generates tests/golden/ref_config0.npz: the reference's own CPU fitter on the
plain-LM workload of 64x64 synthetic texels (81x81 ring directions, RGB FP32,
kd ~ U[0,0.8]^3, ks ~ U[0,1]^3, sigma log-uniform [0.02, 0.8], normal within 30
degrees of +z, x(1 + N(0, 0.01)) noise; the oracle's seeded generator with mix
0), default initial guess.

Run where the reference sources exist (oracle/_ref/libtempest_ref.so is built
from them in place):

    python tests/golden/make_config0_golden.py

For every 16th texel (256 of the 4096) the reference's pipeline
(SVBRDFFitPipeline::cache + fit on a serial pool, so the default initial guess
is deterministic) gives the initial guess, the fit, the RMSE and the iteration
counts.  LeastSquaresFitSGGX caps LM at CurveFitSteps = 1024 iterations
(svbrdf-fitting.hh:51); the iteration counts show where a 100 cap would bind.

    python tests/golden/make_config0_golden.py --full

does the same for all 4096 texels (tests/golden/ref_config0_full.npz; 64-texel
BTFs, one per worker task) and records the wall time and worker count of the
run.
"""
from __future__ import annotations

import multiprocessing as mp
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)

SEED, MIX = 100, 0
SIDE = 64
STEP = 16


def fit_one(t):
    import oracle as O

    tp = O.ring81_angles()
    lp = O.angles_to_parabolic(tp)
    rgb = O.synth_render(SEED, t, O.synth_truth(SEED, MIX, t), lp)
    r = O.RefBTF.from_texels(tp, rgb[None]).fit_texel(0)
    return r["init"], r["fit"], r["rmse"], r["iterations"], r["effective"]


def fit_chunk(first):
    """Texels first .. first+CHUNK-1 as one BTF of CHUNK texels."""
    import oracle as O

    tp = O.ring81_angles()
    lp = O.angles_to_parabolic(tp)
    ts = range(first, first + CHUNK)
    rgb = np.stack([O.synth_render(SEED, t, O.synth_truth(SEED, MIX, t), lp) for t in ts])
    btf = O.RefBTF.from_texels(tp, rgb)
    rows = []
    for x in range(CHUNK):
        r = btf.fit_texel(x)
        rows.append((r["init"], r["fit"], r["rmse"], r["iterations"], r["effective"]))
    return rows


CHUNK = 64


def main():
    import oracle as O

    O.build()
    assert O.ref_available(), "oracle/_ref/libtempest_ref.so was not built (reference sources missing?)"
    full = "--full" in sys.argv[1:]
    workers = os.cpu_count() or 1
    t0 = time.perf_counter()
    if full:
        idx = np.arange(SIDE * SIDE, dtype=np.int64)
        with mp.get_context("spawn").Pool(workers) as pool:
            rows = [r for chunk in pool.map(fit_chunk, list(range(0, SIDE * SIDE, CHUNK))) for r in chunk]
    else:
        idx = np.arange(0, SIDE * SIDE, STEP, dtype=np.int64)
        with mp.get_context("spawn").Pool(workers) as pool:
            rows = pool.map(fit_one, [int(t) for t in idx])
    secs = time.perf_counter() - t0
    init, fit, rmse, it, ef = zip(*rows)
    extra = dict(wall_seconds=secs, workers=workers) if full else {}
    np.savez(os.path.join(HERE, "ref_config0_full.npz" if full else "ref_config0.npz"), seed=SEED, mix=MIX,
             side=SIDE, idx=idx, init=np.asarray(init, np.float32), fit=np.asarray(fit, np.float32),
             rmse=np.asarray(rmse, np.float32), iterations=np.asarray(it, np.uint32),
             effective=np.asarray(ef, np.uint32), **extra)
    print(f"{len(idx)} texels in {secs:.0f} s on {workers} workers: mean rmse {np.mean(rmse):.4e}, "
          f"iterations max {max(it)}, above 100: {sum(i > 100 for i in it)}")


if __name__ == "__main__":
    main()
