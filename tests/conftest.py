import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


@pytest.fixture(scope="session")
def params_all():
    from cltem_b200.params import read_params_json, default_bundle_path
    return read_params_json(default_bundle_path())


@pytest.fixture(scope="session")
def kirkland(params_all):
    return params_all["kirkland"]


@pytest.fixture(scope="session")
def lobato(params_all):
    return params_all["lobato"]


@pytest.fixture(scope="session")
def peng(params_all):
    return params_all["peng"]


@pytest.fixture(scope="session")
def oracle():
    from oracle import bind
    bind.lib()
    return bind


@pytest.fixture(scope="session")
def gpu_ctx():
    """A device context on cuda:0 (GPU tests only)."""
    from cltem_b200.engine import Context
    ctx = Context(0)
    yield ctx
    ctx.close()
