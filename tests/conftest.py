import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


def pytest_collection_modifyitems(config, items):
    # Files are collected in name order; keep it explicit so that
    # test_zz_* files always run last.
    items.sort(key=lambda it: (os.path.basename(str(it.fspath)).startswith("test_zz_"), 0))
