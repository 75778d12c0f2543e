import importlib
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')


def load_package():
    """The engine package; its directory name is not an identifier, so import it by string."""
    return importlib.import_module('bm25-npu_b200')


@pytest.fixture(scope='session')
def pkg():
    return load_package()


@pytest.fixture(scope='session')
def oracle_mod():
    from oracle import oracle
    if not oracle.ORACLE_SO.exists():
        oracle.build(with_reference=False)
    return oracle


@pytest.fixture(scope='session')
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return True
