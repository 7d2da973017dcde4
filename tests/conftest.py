import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# The reference checkout: $GRAPH_RENDER_REFERENCE, else a `reference` directory
# beside this repository. Tests that read it skip when it is absent.
REFERENCE = os.environ.get("GRAPH_RENDER_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running case")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the oracle and the native libraries once per session."""
    from oracle import oracle as O
    from graph_render_b200 import build

    O.build()
    build.build_all()
    yield


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False
