"""The oracle's restatement of the multi-scattering model (svbrdffit -m) against
the reference's own runs (tests/golden/ref_ms.npz, made by make_ms_golden.py from
oracle/_ref): BRDFEvaluator with BounceCount over SGGXMicroFlakePseudoVolumeBRDF
(svbrdf-lsq-fitting-internal.hh:91-153, ggx-models-impl.hh:621-758), and
LeastSquaresFitSGGX with MultiScatteringBounceCount (svbrdf-lsq-fitting-setup.cc:
234-431) -- bit for bit: the same float operations in the same order, the same
LCG sequence (the reference's GCC build draws UniformSampleSphere's second
argument first), glibc's logf/expf/tanf on both sides.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle
import tempestrenderer_b200 as svf


@pytest.fixture(scope="module")
def ms():
    return np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_ms.npz"))


def test_pseudo_volume_brdf_is_bit_exact(ms):
    for i, p in enumerate(ms["params"]):
        for j, b in enumerate(ms["bounces"]):
            got = oracle.brdf_all_ms(p, ms["fib32"], int(b))
            assert np.array_equal(got.view(np.uint32), ms["brdf_fib32"][i, j].view(np.uint32)), (i, int(b))
    got = oracle.brdf_all_ms(ms["params"][0], ms["ring81"], 2)
    assert np.array_equal(got.view(np.uint32), ms["brdf_ring81"].view(np.uint32))


def test_multiple_scattering_adds_energy(ms):
    """More bounces add non-negative walk contributions over the single-scattering
    term (0 bounces), pair by pair, with the same random sequence."""
    p = ms["params"][0]
    e0 = oracle.brdf_all_ms(p, ms["fib32"], 0)
    single = oracle.brdf_all(p, ms["fib32"])[0]
    for b in (1, 2, 4):
        assert (oracle.brdf_all_ms(p, ms["fib32"], b) >= e0).all()
    # the pseudo volume's first term is the surface BRDF's (Fresnel 1) up to rounding
    np.testing.assert_allclose(e0, single, rtol=1e-5, atol=1e-7)


def test_multi_scattering_fit_is_bit_exact(ms):
    for t in range(len(ms["fit_out"])):
        out, rmse, st = oracle.lsq_fit_ms(ms["fit_lum"][t], ms["fib16"], ms["fit_init"][t], int(ms["fit_bounces"]))
        assert np.array_equal(out, ms["fit_out"][t]), t
        assert np.float32(rmse) == ms["fit_rmse"][t]
        assert (st.iterations, st.effective) == tuple(ms["fit_iters"][t])


def test_options_default_and_layout():
    o = svf.LsqOptions()
    svf.load().svf_lsq_options_default(C.byref(o))
    assert o.multi_scattering_bounces == 2 and not (o.flags & svf.SVF_LSQ_MULTI_SCATTERING)
    m = svf.options(multi_scattering=4)
    assert m.flags & svf.SVF_LSQ_MULTI_SCATTERING and m.multi_scattering_bounces == 4
    assert C.sizeof(svf.LsqOptions) == 48
