"""Generates tests/golden/ref_options.npz: the reference's own LeastSquaresFitSGGX
(svbrdf-lsq-fitting-setup.cc:234-431) with the LeastSquaresFitOptions that
svbrdffit exposes beyond the default fit, on the golden texels of
ref_pipeline.npz (seed 11, mix 1, ring-81), from perturbed ground truth:

* specular -- without LSF_OPTON_DIFFUSE: the 6-parameter specular fit
  (BRDFEvaluatorSpecular, AcceptStepSpecularConstraints; diffuse reported 0);
* nodir -- LSF_OPTON_DIFFUSE | LSF_OPTION_DISABLE_DIRECTION_FITTING: the Euler
  angles held (fit_params_count - 3, :265-268);
* specular_nodir -- both;
* down41 -- DownSampleLightView = 41 (svbrdffit -S 41): the 41 x 41 pairs of
  the directions DownsampleLightView keeps (:129-163, :314-330), RMSE over all
  81 x 81 pairs at Fresnel 1 (:403-421);
* top -- LSF_OPTON_DIFFUSE | LSF_OPTION_FIT_TOP: the 81 samples of the top-most
  view (:289-313), RMSE over all pairs at Fresnel 1;

and DownsampleLightView's kept directions for n = 20, 41, 60 (dirs_<n>).  (At 81
directions the reference divides by zero for n = 40, 76 and 79: in float, the
stride end of its next-to-last draw already reaches 81, so the last stride is
empty; svf_downsample_light_view rejects those sizes.)

Run where the reference sources exist (oracle/_ref is built from them in place):

    python tests/golden/make_options_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle as O  # noqa: E402

SEED, MIX, TEXELS = 11, 1, 8
CASES = {"specular": (0, 0xFFFFFFFF),
         "nodir": (O.LSF_OPTON_DIFFUSE | O.LSF_OPTION_DISABLE_DIRECTION_FITTING, 0xFFFFFFFF),
         "specular_nodir": (O.LSF_OPTION_DISABLE_DIRECTION_FITTING, 0xFFFFFFFF),
         "down41": (O.LSF_OPTON_DIFFUSE, 41),
         "top": (O.LSF_OPTON_DIFFUSE | O.LSF_OPTION_FIT_TOP, 0xFFFFFFFF)}


def main():
    O.build()
    assert O.ref_available(), "oracle/_ref/libtempest_ref.so was not built (reference sources missing?)"
    lp = O.angles_to_parabolic(O.ring81_angles())
    truths = [O.truth_lum_params(O.synth_truth(SEED, MIX, t)) for t in range(TEXELS)]
    lum = np.stack([O.lum_slice(O.synth_render(SEED, t, O.synth_truth(SEED, MIX, t), lp))[0] for t in range(TEXELS)])
    rng = np.random.default_rng(23)
    init = []
    for t in truths:
        p = (t * (1 + 0.2 * rng.standard_normal(7))).astype(np.float32)
        p[:4] = np.abs(p[:4]) + 1e-3
        init.append(p)
    init = np.asarray(init, np.float32)
    out = {"seed": SEED, "mix": MIX, "lum": lum, "init": init}
    for name, (flags, down) in CASES.items():
        fits, rmses, iters = [], [], []
        for x in range(TEXELS):
            f, r, it, ef = O.ref_lsq_opts(lum[x], lp, init[x], flags=flags, downsample=down)
            fits.append(f)
            rmses.append(r)
            iters.append((it, ef))
        out[f"{name}_flags"] = flags
        out[f"{name}_downsample"] = down
        out[f"{name}_fit"] = np.asarray(fits)
        out[f"{name}_rmse"] = np.asarray(rmses, np.float32)
        out[f"{name}_iters"] = np.asarray(iters)
        print(name, "rmse", np.round(out[f"{name}_rmse"], 5), flush=True)
    for n in (20, 41, 60):
        dirs, sl = O.ref_downsample(lum[0], lp, n)
        out[f"dirs_{n}"] = dirs
        out[f"slice_{n}"] = sl
    np.savez(os.path.join(HERE, "ref_options.npz"), **out)
    print("written", os.path.join(HERE, "ref_options.npz"))


if __name__ == "__main__":
    main()
