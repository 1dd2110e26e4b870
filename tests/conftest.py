import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long physics check, run with -m slow")


def pytest_collection_modifyitems(config, items):
    # Slow physics checks are opt-in, like the reference's #[ignore = "slow physics check"].
    if config.getoption("-m") and "slow" in config.getoption("-m"):
        return
    skip = pytest.mark.skip(reason="slow physics check: run with -m slow")
    for item in items:
        if "slow" in item.keywords:
            item.add_marker(skip)
