import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libpimdal_b200.so")


@pytest.fixture(scope="session")
def ctx():
    """One pimdal context on cuda:0 for the whole GPU session."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pimdal_b200 import ops
    c = ops.Context(0)
    yield c
    c.close()
