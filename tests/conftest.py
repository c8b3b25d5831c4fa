import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def geometry():
    from allen_b200 import _native
    return _native.default_geometry()


@pytest.fixture(scope="session")
def oracle():
    import cpu_checkers
    if not cpu_checkers.available("oracle"):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "oracle"], check=True)
    return cpu_checkers.load("oracle")


@pytest.fixture(scope="session")
def chain():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from allen_b200.chain import VeloChain
    c = VeloChain()
    yield c
    c.close()
