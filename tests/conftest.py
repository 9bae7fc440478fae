import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")


def params_dict(**kw):
    """StereoParams defaults (include/stereo/stereo_params.h:57-82) as a dict."""
    d = dict(minDisparity=0, maxDisparity=128, blockSize=5, P1=200, P2=800, preFilterCap=31,
             uniquenessRatio=10, disp12MaxDiff=1, speckleWindowSize=100, speckleRange=32,
             useGPU=1, useSharedMemory=1, numDirections=4, matchingCostMode=0)
    d.update(kw)
    return d


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    oracle.lib()
    return oracle
