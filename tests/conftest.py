import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "mille-feuille_b200"), os.path.join(ROOT, "oracle"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle.so")):
        oracle.build()
    return oracle


@pytest.fixture(scope="session")
def mf():
    """The product package; builds the in-tree library when it is missing."""
    lib = os.path.join(ROOT, "mille-feuille_b200", "millefeuille", "libmillefeuille.so")
    if not os.path.exists(lib):
        import importlib
        build = importlib.import_module("build")
        build.build()
    import millefeuille
    return millefeuille


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
