"""The C-ABI library: it loads, exports every entry point include/svf.h
declares, and its host-only entry points (direction tables, triangulation)
behave; no GPU is needed."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import tempestrenderer_b200 as svf

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_functions():
    text = open(os.path.join(REPO, "include", "svf.h")).read()
    return sorted(set(re.findall(r"\b(svf_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_exports():
    assert _declared_functions() == sorted(svf.EXPORTS)


def test_library_exports_every_declared_function(svf_lib):
    for name in _declared_functions():
        assert hasattr(svf_lib, name), name


def test_abi_version_and_status_strings(svf_lib):
    assert svf_lib.svf_abi_version() == 4
    assert svf_lib.svf_status_string(svf.SVF_EINVAL) == b"invalid argument"


def test_create_without_usable_device_fails_cleanly(svf_lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    assert svf_lib.svf_create(0, C.byref(h)) == svf.SVF_ENODEV
    assert not h.value
    assert svf_lib.svf_last_error()


def test_null_arguments_rejected(svf_lib):
    o = svf.LsqOptions()
    svf_lib.svf_lsq_options_default(C.byref(o))
    assert o.max_iterations == 1024 and o.fresnel == 1.0 and o.flags == svf.SVF_LSQ_DIFFUSE | svf.SVF_LSQ_STEP_PER_PARAMETER
    assert svf_lib.svf_lsq_fit_batch(None, None, 81, None, 0, 1, C.byref(o), None, None, None, None) == svf.SVF_EINVAL
    assert svf_lib.svf_fit_texels(None, None, None, None, None) == svf.SVF_EINVAL


def test_ring81_directions_match_the_reference(golden):
    lp = svf.directions_ring81()
    assert np.array_equal(lp, golden["mesh"]["lights_parabolic"])


def _check_mesh(lp, tri, edges, angles):
    P = lp.astype(np.float64)
    a, b, c = P[tri[:, 0]], P[tri[:, 1]], P[tri[:, 2]]
    orient = (b[:, 0] - a[:, 0]) * (c[:, 1] - a[:, 1]) - (b[:, 1] - a[:, 1]) * (c[:, 0] - a[:, 0])
    assert (orient > 0).all()
    assert len(np.unique(tri)) == lp.shape[0]
    assert (np.diff(angles[:, 1]) >= 0).all()


@pytest.mark.parametrize("layout", ["ring81", "fib151"])
def test_triangulation_is_valid(layout):
    lp = svf.directions_ring81() if layout == "ring81" else svf.directions_fibonacci(151)
    tri, edges, angles = svf.triangulate(lp)
    _check_mesh(lp, tri, edges, angles)
    # Euler: T = 2n - h - 2 for a triangulation of n points with h on the hull
    n, h = lp.shape[0], edges.shape[0]
    assert tri.shape[0] == 2 * n - h - 2


def test_boundary_edges_match_loadbtf(golden):
    """The ring layout's hull is the outer ring, so the boundary edges do not
    depend on how cocircular points were triangulated."""
    m = golden["mesh"]
    tri, edges, angles = svf.triangulate(m["lights_parabolic"])
    assert np.array_equal(edges[:, :2], m["edges"][:, :2])
    assert np.array_equal(angles, m["edge_angles"])
