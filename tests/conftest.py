import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on CPU")


@pytest.fixture(scope="session")
def zs():
    """The product package with its CUDA library loaded (built if missing)."""
    from zsmpm_b200 import build
    build.build()
    import zsmpm_b200
    zsmpm_b200._abi.lib()
    return zsmpm_b200


@pytest.fixture(scope="session")
def gpu(zs):
    if zs.device_count() < 1:
        pytest.fail("a GPU test ran without a visible CUDA device")
    import torch
    torch.cuda.init()
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def reference_cli():
    """The compiled reference (oracle/_ref/zsref_cli).  GPU parity tests compare against it and
    fail when it is missing, rather than compare against the restatement in its place."""
    from oracle import reference
    if not reference.available():
        pytest.fail("oracle/_ref/zsref_cli (the reference compiled by oracle/build_ref.sh) is missing; "
                    "the parity tests that name the reference never fall back to the restatement")
    return reference
