"""svbrdffit -r on the CPU: the fit parameters of saved maps
(svf_params_from_maps), against the oracle's Euler/quaternion restatement and
the reference's own output maps (tests/golden/ref_pipeline.npz): converting the
reference's maps back gives the reference's fitted parameters."""
import numpy as np

import tempestrenderer_b200 as svf


def test_quaternion_to_euler_roundtrip(oracle_lib):
    rng = np.random.default_rng(4)
    for _ in range(200):
        e = rng.uniform(-3, 3, 3).astype(np.float32)
        e[1] = rng.uniform(-1.5, 1.5)
        R, q = oracle_lib.euler_to_matrix(e)
        d = np.ones((1, 3), np.float32)
        p, _ = svf.params_from_maps(d, d, np.array([[0.2, 0.1]], np.float32), q[None])
        R2, _ = oracle_lib.euler_to_matrix(p[0, 4:7])
        np.testing.assert_allclose(R2, R, atol=3e-6)


def test_reference_maps_give_reference_parameters(golden):
    p = golden["pipeline"]
    maps = p["maps"]          # sigma (2), quaternion (4), diffuse (3), specular (3) per texel
    fit = p["fit"]
    avg = p["avg"]
    sigma, quat, diffuse, specular = maps[:, 0:2], maps[:, 2:6], maps[:, 6:9], maps[:, 9:12]
    params, colour = svf.params_from_maps(diffuse, specular, sigma, quat)
    np.testing.assert_array_equal(params[:, 0:2], fit[:, 0:2])
    # the albedos are avg * kd: their luminance is kd up to lum(avg) = 1 and a few ulp of rounding
    np.testing.assert_allclose(params[:, 2], fit[:, 2], rtol=4e-6, atol=1e-9)
    np.testing.assert_allclose(params[:, 3], fit[:, 3], rtol=4e-6, atol=1e-9)
    np.testing.assert_allclose(colour, avg, rtol=4e-6)
    import oracle

    for t in range(len(fit)):
        R, _ = oracle.euler_to_matrix(fit[t, 4:7])
        R2, _ = oracle.euler_to_matrix(params[t, 4:7])
        np.testing.assert_allclose(R2, R, atol=3e-6)
    # three-channel scale maps are divided by their third channel
    s3 = np.concatenate([sigma * 2.0, np.full((len(fit), 1), 2.0, np.float32)], 1)
    p3, _ = svf.params_from_maps(diffuse, specular, s3, quat)
    np.testing.assert_allclose(p3[:, 0:2], fit[:, 0:2], rtol=1e-7)
