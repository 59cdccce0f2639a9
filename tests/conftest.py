import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    if not os.path.exists(oracle.ORACLE_SO):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    d = os.path.join(REPO, "tests", "golden")
    return {
        "mesh": np.load(os.path.join(d, "ring81_mesh.npz")),
        "angles": np.load(os.path.join(d, "ring81_angles.npz"))["theta_phi"],
        "pipeline": np.load(os.path.join(d, "ref_pipeline.npz")),
        "lsq": np.load(os.path.join(d, "ref_lsq.npz")),
    }


@pytest.fixture(scope="session")
def svf_lib():
    import tempestrenderer_b200 as svf

    return svf.load()


@pytest.fixture(scope="session")
def gpu_ctx():
    import tempestrenderer_b200 as svf

    ctx = svf.Context(0)
    yield ctx
    ctx.close()
