"""Generates tests/golden/*.npz from the reference's own CPU fitter.

Run where the reference sources exist (the oracle Makefile compiles them in
place into oracle/_ref/libtempest_ref.so):

    python tests/golden/make_golden.py

Inputs are synthetic texels rendered by the oracle's seeded generator
(svfo_synth_*), written as a DFMF file and loaded through the reference's
LoadBTF; every number stored is produced by the reference build:

* ring81_mesh.npz -- the 81-direction ring layout as LoadBTF stores it
  (LightsParabolic) and the interpolation mesh it builds (LightIndices, Edges).
* ref_pipeline.npz -- per texel: luminance-slice sum, average chromaticity,
  the default initial guess, the LeastSquaresFitSGGX result, RMSE, iteration
  counts, the 64x64 NDF texture and the five output-map values
  (SVBRDFFitPipeline::cache + fit, one worker thread).
* ref_lsq.npz -- LeastSquaresFitSGGX from perturbed ground-truth initial
  guesses, and BRDFEvaluator values for a set of parameter vectors.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402

SEED, MIX = 11, 1
TEXELS = 8


def main():
    O.build()
    assert O.ref_available(), "oracle/_ref/libtempest_ref.so was not built (reference sources missing?)"
    tp = O.ring81_angles()
    lp = O.angles_to_parabolic(tp)
    truths = [O.synth_truth(SEED, MIX, t) for t in range(TEXELS)]
    rgb = np.stack([O.synth_render(SEED, t, truths[t], lp) for t in range(TEXELS)])
    btf = O.RefBTF.from_texels(tp, rgb)
    mesh = btf.mesh()
    assert np.array_equal(mesh.lights_parabolic, lp)
    mesh.save(os.path.join(HERE, "ring81_mesh.npz"))
    np.savez(os.path.join(HERE, "ring81_angles.npz"), theta_phi=tp)

    rec = {k: [] for k in ("lum_sum", "avg", "init", "fit", "rmse", "iterations", "effective", "ndf", "maps",
                           "truth")}
    for x in range(TEXELS):
        lum, avg = btf.lum_slice(x)
        r = btf.fit_texel(x, want_ndf=True)
        rec["lum_sum"].append(float(np.sum(lum, dtype=np.float64)))
        rec["avg"].append(avg)
        rec["init"].append(r["init"])
        rec["fit"].append(r["fit"])
        rec["rmse"].append(r["rmse"])
        rec["iterations"].append(r["iterations"])
        rec["effective"].append(r["effective"])
        rec["ndf"].append(r["ndf"])
        rec["maps"].append(r["maps"])
        rec["truth"].append(O.truth_lum_params(truths[x]))
        print(f"texel {x}: rmse {r['rmse']:.3e} iterations {r['iterations']} ({r['effective']})", flush=True)
    np.savez(os.path.join(HERE, "ref_pipeline.npz"), seed=SEED, mix=MIX,
             **{k: np.asarray(v) for k, v in rec.items()})

    # LeastSquaresFitSGGX from perturbed ground truth
    rng = np.random.default_rng(5)
    inits, fits, rmses, iters = [], [], [], []
    for x in range(TEXELS):
        lum, _ = btf.lum_slice(x)
        t = O.truth_lum_params(truths[x])
        init = (t * (1 + 0.2 * rng.standard_normal(7))).astype(np.float32)
        init[:4] = np.abs(init[:4]) + 1e-3
        out, rmse, it, ef = O.ref_lsq(lum, lp, init)
        inits.append(init)
        fits.append(out)
        rmses.append(rmse)
        iters.append((it, ef))
    # BRDFEvaluator on every 7th pair for a few parameter vectors
    params = np.array([[0.3, 0.1, 0.8, 0.4, 0.2, -0.1, 0.7],
                       [0.05, 0.6, 0.2, 0.1, -0.3, 0.25, -1.2],
                       [0.02, 0.02, 1.0, 0.0, 0.0, 0.0, 0.0],
                       [0.8, 0.7, 0.05, 0.6, 0.4, 0.4, 2.5],
                       [-0.1, 0.3, -0.2, 0.5, 0.1, 0.2, 0.3]], np.float64)
    pairs = np.arange(0, 81 * 81, 7, dtype=np.int64)
    brdf = np.stack([O.ref_brdf_all(p, lp)[pairs] for p in params])
    np.savez(os.path.join(HERE, "ref_lsq.npz"), init=np.asarray(inits), fit=np.asarray(fits),
             rmse=np.asarray(rmses), iters=np.asarray(iters), brdf_params=params, brdf_pairs=pairs, brdf=brdf)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
