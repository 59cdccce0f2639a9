"""svf_downsample_light_view -- the library's restatement of the direction choice
of DownsampleLightView (svbrdf-lsq-fitting-setup.cc:129-163) -- against the
reference's own (tests/golden/ref_options.npz, tests/golden/make_options_golden.py):
the kept directions and the downsampled slice, bit for bit.  At 81 directions
the reference divides by zero for n = 40, 76 and 79 (an empty last stride); the
library rejects those sizes instead.  No GPU is needed."""
import os

import numpy as np
import pytest

import tempestrenderer_b200 as svf

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def opts_golden():
    return np.load(os.path.join(HERE, "golden", "ref_options.npz"))


@pytest.mark.parametrize("n", [20, 41, 60])
def test_downsample_directions_match_reference(golden, opts_golden, n):
    lp = golden["mesh"]["lights_parabolic"]
    idx = svf.downsample_light_view(81, n)
    assert np.array_equal(lp[idx], opts_golden[f"dirs_{n}"])
    lum = opts_golden["lum"][0]
    sub = lum.reshape(81, 81)[np.ix_(idx, idx)].reshape(-1)
    assert np.array_equal(sub, opts_golden[f"slice_{n}"])


@pytest.mark.parametrize("n", [40, 76, 79, 1, 81, 0])
def test_downsample_sizes_without_a_draw_are_rejected(n):
    with pytest.raises(svf.SvfError):
        svf.downsample_light_view(81, n)
