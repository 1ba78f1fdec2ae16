import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built nozomi_b200 library")
    config.addinivalue_line("markers", "slow: longer statistical runs")


def pytest_collection_modifyitems(config, items):
    # GPU tests never run silently on a machine without a GPU: they fail loudly
    # there if selected explicitly, and are deselected by -m "not gpu".
    pass
