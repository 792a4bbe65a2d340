import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(TESTS, "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests proper")


@pytest.fixture(scope="session")
def nb():
    import necpp_b200
    return necpp_b200


@pytest.fixture(scope="session")
def api(nb):
    class API:
        def __getattr__(self, k):
            return getattr(nb, k)

        def helix(self, ctx, *a):
            return nb.nec_helix(ctx, *a)

    return API()


@pytest.fixture(scope="session")
def oracle():
    from oracle.momwrap import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def ref():
    from oracle import refwrap
    if not refwrap.available():
        pytest.skip("reference build oracle/_ref not present on this host")
    return refwrap.RefAPI()


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
