"""Generates tests/golden/ref_fresnel.npz from the reference's own CPU fitter at
svbrdffit's default refractive index, 1.5 (svbrdf-fitting.cc:193,262), where the
surface BRDF carries the dielectric Fresnel factor (ggx-models-impl.hh:525-536,
FresnelDielectric, functions.hh:296-301).

Run where the reference sources exist (oracle/_ref/libtempest_ref.so is built
from them in place):

    python tests/golden/make_fresnel_golden.py

Every number stored is produced by the reference build:

* brdf -- BRDFEvaluator values at Fresnel 1.5 on every 7th pair for the
  parameter vectors of ref_lsq.npz.
* texels -- 8 luminance slices rendered by the reference's BRDFEvaluator at
  Fresnel 1.5 from seeded ground truth (the oracle's synthetic generator), times
  (1 + 0.01 N(0, 1)) seeded noise; the LeastSquaresFitSGGX result at Fresnel
  1.5 from perturbed ground truth (lsq_*); and the full pipeline
  (SVBRDFFitPipeline::cache + fit, one worker thread) on the same slices as a
  grey RGB BTF loaded through LoadBTF (pipe_*: default initial guess, fit,
  RMSE, iterations).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402

FRESNEL = 1.5
SEED, MIX = 17, 1
TEXELS = 8


def fresnel_texels(lp):
    """Luminance slices rendered at Fresnel 1.5 by the reference's evaluator."""
    rng = np.random.default_rng(SEED)
    truth, lum = [], []
    for x in range(TEXELS):
        t = O.truth_lum_params(O.synth_truth(SEED, MIX, x)).astype(np.float64)
        f = O.ref_brdf_all(t, lp, FRESNEL).astype(np.float64)
        y = f * (1.0 + 0.01 * rng.standard_normal(f.shape))
        truth.append(t)
        lum.append(y.astype(np.float32))
    return np.asarray(truth, np.float32), np.asarray(lum, np.float32)


def main():
    O.build()
    assert O.ref_available(), "oracle/_ref/libtempest_ref.so was not built (reference sources missing?)"
    tp = O.ring81_angles()
    lp = O.angles_to_parabolic(tp)
    lsq = np.load(os.path.join(HERE, "ref_lsq.npz"))
    params, pairs = lsq["brdf_params"], lsq["brdf_pairs"]
    brdf = np.stack([O.ref_brdf_all(p, lp, FRESNEL)[pairs] for p in params])

    truth, lum = fresnel_texels(lp)
    rng = np.random.default_rng(SEED + 1)
    rec = {k: [] for k in ("lsq_init", "lsq_fit", "lsq_rmse", "lsq_iters")}
    for x in range(TEXELS):
        init = (truth[x] * (1 + 0.2 * rng.standard_normal(7))).astype(np.float32)
        init[:4] = np.abs(init[:4]) + 1e-3
        out, rmse, it, ef = O.ref_lsq(lum[x], lp, init, fresnel=FRESNEL)
        rec["lsq_init"].append(init)
        rec["lsq_fit"].append(out)
        rec["lsq_rmse"].append(rmse)
        rec["lsq_iters"].append((it, ef))

    # the pipeline on the slices as a grey RGB BTF (luminance of (g, g, g) is g)
    rgb = np.repeat(lum[:, :, None], 3, axis=2)
    btf = O.RefBTF.from_texels(tp, rgb)
    pipe = {k: [] for k in ("pipe_lum", "pipe_init", "pipe_fit", "pipe_rmse", "pipe_iterations")}
    for x in range(TEXELS):
        sl, _ = btf.lum_slice(x)
        r = btf.fit_texel(x, fresnel=FRESNEL)
        pipe["pipe_lum"].append(sl)
        pipe["pipe_init"].append(r["init"])
        pipe["pipe_fit"].append(r["fit"])
        pipe["pipe_rmse"].append(r["rmse"])
        pipe["pipe_iterations"].append(r["iterations"])
        print(f"texel {x}: lsq rmse {rec['lsq_rmse'][x]:.3e}, pipeline rmse {r['rmse']:.3e} "
              f"({r['iterations']} iterations)", flush=True)
    np.savez(os.path.join(HERE, "ref_fresnel.npz"), fresnel=FRESNEL, seed=SEED, mix=MIX, brdf_params=params,
             brdf_pairs=pairs, brdf=brdf, truth=truth, lum=lum,
             **{k: np.asarray(v) for k, v in {**rec, **pipe}.items()})
    print("written", os.path.join(HERE, "ref_fresnel.npz"))


if __name__ == "__main__":
    main()
