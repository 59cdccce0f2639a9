"""Factored BTF files (DFMF, FMF0, FMF1) on the CPU: the oracle's decode and
the library's host parser (svf_btf_probe) against what the reference's own
LoadBTF / BTFFetchSpectrum did with the same files (tests/golden/ref_btf.npz,
made by tests/golden/make_btf_golden.py from the reference build)."""
import numpy as np
import pytest

import tempestrenderer_b200 as svf

FMT = {0: "DFMF", 1: "FMF0", 2: "FMF1"}


@pytest.fixture(scope="module")
def ref_btf():
    import os

    return np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_btf.npz"))


def _cases(ref_btf, accepted):
    return [str(n) for n in ref_btf["names"] if bool(ref_btf[f"{n}/ok"]) == accepted]


def test_probe_accepts_what_loadbtf_accepts(ref_btf):
    for name in ref_btf["names"]:
        name = str(name)
        data = ref_btf[f"{name}/bytes"].tobytes()
        if bool(ref_btf[f"{name}/ok"]):
            info, lp = svf.btf_probe(data)
            fmt, ds, cm, drr, W, H, L = (int(v) for v in ref_btf[f"{name}/meta"])
            assert (info.format, info.data_size, info.color_model, info.dynamic_range_reduction) == (fmt, ds, cm, drr)
            assert (info.width, info.height, info.light_count) == (W, H, L)
            # LightsParabolic as LoadBTF derived it, bit for bit
            np.testing.assert_array_equal(lp, ref_btf[f"{name}/lights_parabolic"], err_msg=name)
        else:
            with pytest.raises(svf.SvfError):
                svf.btf_probe(data)


def test_oracle_decode_matches_loadbtf(ref_btf, oracle_lib):
    """The oracle restatement regenerates each golden file's planes from the
    generator's seed and decodes them bit-identically to BTFFetchSpectrum."""
    import sys
    import os

    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_btf_golden as G

    for name, fmt, ds, cm, drr, data in G.cases():
        if not bool(ref_btf[f"{name}/ok"]):
            continue
        assert data == ref_btf[f"{name}/bytes"].tobytes(), name   # the generator is deterministic
        planes = G.case_planes(name)
        got = oracle_lib.btf_decode(planes, fmt, G.W, G.H, G.L, ds, cm, drr)
        ref = ref_btf[f"{name}/spectra"]
        np.testing.assert_array_equal(got.view(np.uint32), ref.view(np.uint32), err_msg=name)
