import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ctx():
    from cortexraytracercuda_b200.renderer import Context
    c = Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def refcpu():
    import oracles
    o = oracles.ref_cpu()
    if o is None:
        pytest.skip("oracle/_ref/libref_cpu.so not built")
    return o


@pytest.fixture(scope="session")
def refgpu():
    import oracles
    o = oracles.ref_gpu()
    if o is None:
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    return o
