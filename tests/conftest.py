"""Shared fixtures: synthetic case files, the oracle, GPU detection."""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


# Small versions of the five workloads, with the build choices the reference
# fixes at compile time (kernel, wall streamer).
SMALL_CASES = {
    # name: (workload, scale, kernel, wall, steps)
    "pipe_r8": ("pipe_r8", 1.0, "LBGK", "SBB", 2000),
    "pipe_bfl": ("pipe_r40", 0.2, "LBGK", "BFL", 1000),
    "bifurcation": ("bifurcation", 0.25, "TRT", "GZS", 1000),
    "stenosis": ("stenosis", 0.2, "LBGKLESSL", "BFL", 1000),
}


@pytest.fixture(scope="session")
def case_dir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("cases"))


_made = {}


def make_small_case(case_dir, key):
    from hemepure_b200 import vessels
    if key not in _made:
        workload, scale, kernel, wall, steps = SMALL_CASES[key]
        d = os.path.join(case_dir, key)
        xml, gmy, info = vessels.make_case(workload, d, steps=steps, scale=scale)
        _made[key] = (xml, gmy, info, kernel, wall, steps)
    return _made[key]


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
