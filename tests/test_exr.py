"""svbrdffit's OpenEXR map files on the CPU: the library reads what the
reference's SaveEXRImage wrote (tests/golden/ref_error.npz, from
tests/golden/make_error_golden.py), its own files round-trip, and -- where the
reference build is present -- the reference's LoadEXRImage reads the library's
files back to the same pixels."""
import os
import tempfile

import numpy as np
import pytest

import tempestrenderer_b200 as svf


@pytest.fixture(scope="module")
def ref_error():
    return np.load(os.path.join(os.path.dirname(__file__), "golden", "ref_error.npz"))


def _tmp(suffix=".exr"):
    fd, path = tempfile.mkstemp(suffix=suffix)
    os.close(fd)
    return path


def test_reads_reference_exr(ref_error):
    for c in range(1, 5):
        path = _tmp()
        try:
            open(path, "wb").write(ref_error[f"exr/{c}/bytes"].tobytes())
            img = svf.exr_read(path)
        finally:
            os.unlink(path)
        np.testing.assert_array_equal(img, ref_error[f"exr/{c}/pixels"])


@pytest.mark.parametrize("channels", [1, 2, 3, 4])
def test_roundtrip_and_reference_reads_ours(channels, oracle_lib):
    rng = np.random.default_rng(channels)
    img = rng.normal(0, 3, (9, 13, channels)).astype(np.float32)
    path = _tmp()
    try:
        svf.exr_write(path, img)
        np.testing.assert_array_equal(svf.exr_read(path), img)
        if oracle_lib.ref_available():
            dims = np.zeros(3, np.uint32)
            out = np.zeros(img.size, np.float32)
            assert oracle_lib.ref().ref_exr_load(path.encode(), dims, out.ctypes.data)
            assert tuple(dims) == (13, 9, channels)
            np.testing.assert_array_equal(out.reshape(img.shape), img)
    finally:
        os.unlink(path)


def test_maps_file_set_and_errors(tmp_path):
    rng = np.random.default_rng(3)
    W, H = 5, 4
    maps = {"diffuse": rng.random((H * W, 3), np.float32), "specular": rng.random((H * W, 3), np.float32),
            "sigma": rng.random((H * W, 2), np.float32), "basis": rng.random((H * W, 4), np.float32),
            "rmse": rng.random(H * W, dtype=np.float32)}
    prefix = str(tmp_path / "fit")
    svf.maps_write_exr(prefix, W, H, maps)
    for suffix, key in (("albedo", "diffuse"), ("specular", "specular"), ("sggx_scale", "sigma"),
                        ("sggx_basis", "basis"), ("rmse", "rmse")):
        img = svf.exr_read(f"{prefix}_{suffix}.exr")
        np.testing.assert_array_equal(img.reshape(H * W, -1), maps[key].reshape(H * W, -1))
    bad = tmp_path / "bad.exr"
    bad.write_bytes(b"not an exr file")
    with pytest.raises(svf.SvfError):
        svf.exr_read(str(bad))
    with pytest.raises(svf.SvfError):
        svf.exr_write(str(tmp_path / "x.exr"), np.zeros((2, 2, 5), np.float32))
