import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
LN2 = 0.6931471805599453


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (B200)")


@pytest.fixture(scope="session")
def ref32():
    from oracle.ref import RefEngine, available
    if not available(32):
        pytest.fail("oracle/_ref/libdmst_ref32.so missing: run `make -C oracle` (the reference oracle)")
    e = RefEngine(32)
    e.set_rates()
    return e


@pytest.fixture(scope="session")
def ref64():
    from oracle.ref import RefEngine, available
    if not available(64):
        pytest.fail("oracle/_ref/libdmst_ref64.so missing: run `make -C oracle`")
    e = RefEngine(64)
    e.set_rates()
    return e


@pytest.fixture(scope="session")
def regression():
    return dict(np.load(os.path.join(GOLDEN, "regression.npz")))


@pytest.fixture(scope="session")
def gpu_ctx():
    import dummest_b200 as d
    ctx = d.Context(device=0)
    yield ctx
    ctx.close()
