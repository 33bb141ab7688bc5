import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# Every contract! output starts as NaN in the tests, so an element that no
# kernel writes fails the comparisons instead of passing on stale memory.
os.environ.setdefault("SPARSEB_POISON_OUTPUT", "1")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 GPU (sm_100a)")
