import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "sitk-rs_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libmi_b200.so")


def _has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


def geo_dict(size, spacing=(1.0, 1.0, 1.0), origin=(0.0, 0.0, 0.0),
             direction=(1, 0, 0, 0, 1, 0, 0, 0, 1)):
    return {"size": list(size), "spacing": list(spacing), "origin": list(origin),
            "direction": list(direction)}


def small_pair(n=20, seed=7, nblobs=6, rot=8.0, trans=3.0, scale=(0.95, 1.05)):
    from sitk_b200 import synth
    return synth.make_pair(n, nblobs, seed, rot, trans, scale)
