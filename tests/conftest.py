import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine's kernels")
    config.addinivalue_line("markers", "slow: large inputs (seconds of CPU work)")


@pytest.fixture(scope="session")
def db():
    """One GPU context for the whole session (tables are replaced per test)."""
    import falcondb_b200 as F

    d = F.Database(0)
    yield d
    d.close()
