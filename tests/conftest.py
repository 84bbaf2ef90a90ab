"""Test configuration: import paths, the `gpu` marker, shared fixtures."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "alto-stream_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        have_gpu = torch.cuda.is_available()
    except Exception:
        have_gpu = False
    if have_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def load_fixture(name):
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return d["dims"].astype(np.uint64), d["cidx"].astype(np.uint64), d["vals"].astype(np.float64)


def load_stream_fixture():
    d = np.load(os.path.join(GOLDEN, "stream_small.npz"))
    n = len([k for k in d.files if k.startswith("dims")])
    return [dict(dims=d[f"dims{s}"], cidx=d[f"cidx{s}"], vals=d[f"vals{s}"]) for s in range(n)]


FIXTURE_NAMES = ["small", "small4", "small4_zeroidx", "med", "med4", "med5"]
