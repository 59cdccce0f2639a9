"""Pins the oracle restatement's Fresnel branch against the reference at
svbrdffit's default refractive index 1.5 (svbrdf-fitting.cc:193,262;
ggx-models-impl.hh:525-536, FresnelDielectric functions.hh:296-301).

tests/golden/ref_fresnel.npz was produced by the reference's own CPU fitter
(tests/golden/make_fresnel_golden.py).  The restatement keeps the reference's
float operation order, so the comparisons are exact.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def fres():
    return np.load(os.path.join(HERE, "golden", "ref_fresnel.npz"))


def _mesh(oracle, golden):
    m = golden["mesh"]
    return oracle.MeshData(m["lights_parabolic"], m["triangles"], m["edges"], m["edge_angles"])


def test_fresnel_brdf_evaluator_exact(oracle_lib, golden, fres):
    lp = golden["mesh"]["lights_parabolic"]
    F = float(fres["fresnel"])
    assert F == 1.5
    for params, ref, ref1 in zip(fres["brdf_params"], fres["brdf"], golden["lsq"]["brdf"]):
        f32, f64 = oracle_lib.brdf_all(params, lp, F)
        assert np.array_equal(f32[fres["brdf_pairs"]], ref)
        np.testing.assert_allclose(f64[fres["brdf_pairs"]], ref, rtol=2e-5, atol=1e-7)
        # the Fresnel factor lowers the specular term (dielectric reflectance < 1)
        assert np.all(ref <= ref1 + 1e-7)


@pytest.mark.parametrize("x", range(8))
def test_fresnel_lsq_from_perturbed_truth_exact(oracle_lib, golden, fres, x):
    lp = golden["mesh"]["lights_parabolic"]
    out, rmse, st = oracle_lib.lsq_fit(fres["lum"][x], lp, fres["lsq_init"][x], fresnel=1.5)
    assert np.array_equal(out, fres["lsq_fit"][x])
    assert np.float32(rmse) == np.float32(fres["lsq_rmse"][x])
    assert (st.iterations, st.effective) == tuple(fres["lsq_iters"][x])


@pytest.mark.parametrize("x", [0, 2, 5])
def test_fresnel_pipeline_exact(oracle_lib, golden, fres, x):
    """Grey RGB samples: the luminance slice, the default initial guess (which does
    not depend on the Fresnel factor) and the Fresnel LM equal the reference's."""
    lp = golden["mesh"]["lights_parabolic"]
    rgb = np.repeat(fres["lum"][x][:, None], 3, axis=1)
    lum, _ = oracle_lib.lum_slice(rgb)
    assert np.array_equal(lum, fres["pipe_lum"][x])
    init, _ = oracle_lib.default_init_from_ndf(oracle_lib.ndf_texture(_mesh(oracle_lib, golden), lum))
    assert np.array_equal(init, fres["pipe_init"][x])
    out, rmse, st = oracle_lib.lsq_fit(lum, lp, init, fresnel=1.5)
    assert np.array_equal(out, fres["pipe_fit"][x])
    assert np.float32(rmse) == np.float32(fres["pipe_rmse"][x])
    assert st.iterations == fres["pipe_iterations"][x]
