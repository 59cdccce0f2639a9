"""Generates tests/golden/ref_ms.npz: the reference's own multi-scattering model
(BRDFEvaluator with BounceCount = bounces, svbrdf-lsq-fitting-internal.hh:91-153,
over SGGXMicroFlakePseudoVolumeBRDF, ggx-models-impl.hh:621-758) and its
LeastSquaresFitSGGX with LeastSquaresFitOptions::MultiScatteringBounceCount
(svbrdffit -m), run from oracle/_ref (the reference compiled in place):

* brdf_fib32: the evaluator over the 32 x 32 pairs of the 32-direction
  Fibonacci layout, for 4 parameter vectors (params) and bounces 1, 2, 4;
* brdf_ring81: the evaluator over the 81 x 81 ring-81 pairs, params[0], bounces 2;
* fit_*: LeastSquaresFitSGGX with bounces 2 on the 16-direction Fibonacci layout
  for 6 texels: slices rendered by the pseudo-volume model from ground truth
  (the oracle's restatement, pinned above) plus seeded noise, started from
  perturbed ground truth.

Run where the reference sources exist:

    python tests/golden/make_ms_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402
import tempestrenderer_b200 as svf  # noqa: E402

PARAMS = np.array([[0.30, 0.20, 0.80, 0.10, 0.20, -0.10, 0.30],
                   [0.08, 0.15, 1.20, 0.05, -0.30, 0.25, 1.10],
                   [0.45, 0.40, 0.50, 0.30, 0.05, 0.40, -0.70],
                   [0.03, 0.05, 2.00, 0.00, 0.10, 0.10, 0.00]])
BOUNCES = (1, 2, 4)
FIT_TEXELS, FIT_BOUNCES = 6, 2


def main():
    O.build()
    assert O.ref_available(), "oracle/_ref/libtempest_ref.so was not built (reference sources missing?)"
    fib32 = svf.directions_fibonacci(32)
    fib16 = svf.directions_fibonacci(16)
    ring81 = O.angles_to_parabolic(O.ring81_angles())
    out = {"params": PARAMS, "bounces": np.array(BOUNCES), "fib32": fib32, "fib16": fib16, "ring81": ring81}
    out["brdf_fib32"] = np.stack([np.stack([O.ref_brdf_all_ms(p, fib32, b) for b in BOUNCES]) for p in PARAMS])
    out["brdf_ring81"] = O.ref_brdf_all_ms(PARAMS[0], ring81, 2)
    rng = np.random.default_rng(31)
    truth, lum, init = [], [], []
    for t in range(FIT_TEXELS):
        p = np.array([0.05 + 0.4 * rng.random(), 0.05 + 0.4 * rng.random(), 0.4 + 1.2 * rng.random(),
                      0.3 * rng.random(), *(0.8 * (rng.random(3) - 0.5))])
        sl = O.brdf_all_ms(p, fib16, FIT_BOUNCES)
        sl = (sl * (1.0 + 0.01 * rng.standard_normal(sl.shape))).astype(np.float32)
        q = (p * (1 + 0.15 * rng.standard_normal(7))).astype(np.float32)
        q[:4] = np.abs(q[:4]) + 1e-3
        truth.append(p)
        lum.append(sl)
        init.append(q)
    fits, rmses, iters = [], [], []
    for t in range(FIT_TEXELS):
        f, r, it, ef = O.ref_lsq_ms(lum[t], fib16, init[t], FIT_BOUNCES)
        fits.append(f)
        rmses.append(r)
        iters.append((it, ef))
        print("texel", t, "rmse", r, "iterations", it, ef, flush=True)
    out.update(fit_truth=np.asarray(truth), fit_lum=np.asarray(lum), fit_init=np.asarray(init),
               fit_out=np.asarray(fits), fit_rmse=np.asarray(rmses, np.float32), fit_iters=np.asarray(iters),
               fit_bounces=FIT_BOUNCES)
    np.savez_compressed(os.path.join(HERE, "ref_ms.npz"), **out)
    print("written", os.path.join(HERE, "ref_ms.npz"))


if __name__ == "__main__":
    main()
