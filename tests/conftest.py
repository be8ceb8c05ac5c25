import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "latticematrices.jl_b200"),
          os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line(
        "markers", "gpu: needs a CUDA device (B200) and the built liblmb200.so")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as orc_mod
    orc_mod.lib()
    return orc_mod
