import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200)")


@pytest.fixture(scope="session")
def engine():
    from rsr_b200.evaluator import Engine
    e = Engine()
    yield e
    e.close()


@pytest.fixture(scope="session")
def plain_engine():
    from rsr_b200 import _native as N
    from rsr_b200.evaluator import Engine
    e = Engine(kernel=N.KERNEL_PLAIN)
    yield e
    e.close()
