import json
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_masked():
    with open(os.path.join(GOLDEN, "golden_masked.json")) as f:
        return json.load(f)["masked"]


@pytest.fixture(scope="session")
def golden_colour():
    with open(os.path.join(GOLDEN, "golden_colour.json")) as f:
        return json.load(f)["colour"]


@pytest.fixture(scope="session")
def golden_ssim_modes():
    with open(os.path.join(GOLDEN, "golden_ssim_modes.json")) as f:
        return json.load(f)["ssim_modes"]


@pytest.fixture(scope="session")
def cps_arrays():
    import numpy as np
    return dict(np.load(os.path.join(GOLDEN, "cps_fixtures.npz")))


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    return oracle.Oracle()


@pytest.fixture(scope="session")
def qctx():
    if not cuda_available():
        pytest.skip("no CUDA device")
    import qmiv_b200
    ctx = qmiv_b200.Context(0)
    yield ctx
    ctx.close()
