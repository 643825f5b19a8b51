import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "tests", "golden")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def have_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # noqa: BLE001
        return False


@pytest.fixture(scope="session")
def gpu():
    if not have_gpu():
        pytest.fail("this test needs a CUDA GPU")
    return True


@pytest.fixture(autouse=True)
def _ibm_env():
    """The reference reads IBM_BETA / IBM_RAMP_STEPS from the environment on
    every velocity step (src/fluid.cu:199, :266) and oracle/pyref.py sets them;
    restore both after each test so that no test sees another's settings."""
    saved = {k: os.environ.get(k) for k in ("IBM_BETA", "IBM_RAMP_STEPS")}
    yield
    for k, v in saved.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
