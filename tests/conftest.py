import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (run with -m gpu on a B200)")
    config.addinivalue_line("markers", "slow: takes more than a few seconds on the CPU")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.lib()
    return O


@pytest.fixture(scope="session")
def native():
    sys.path.insert(0, ROOT)
    import onion_gen_b200 as og

    return og


@pytest.fixture(scope="session")
def device(native):
    devs = native.gpu.look()
    if not devs:
        pytest.fail("no CUDA device: the gpu tests need a B200")
    return devs[0]
