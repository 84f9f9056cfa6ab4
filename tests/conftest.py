import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200, sm_100a) and the built "
        "libd3d_b200.so")
    config.addinivalue_line(
        "markers", "ref: needs oracle/_ref (the reference objects built from "
        "the reference sources)")


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_cuda():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        meta = json.load(f)
    fields = np.load(os.path.join(GOLDEN_DIR, "fields.npz"))
    return meta, fields


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def golden_diffusion():
    """Fixtures of the diffusion::Diffusion surface (2D and 3D grids)."""
    with open(os.path.join(GOLDEN_DIR, "diffusion.json")) as f:
        meta = json.load(f)
    fields = np.load(os.path.join(GOLDEN_DIR, "diffusion_fields.npz"))
    return meta, fields
