"""Shared test set-up.

Markers: ``gpu`` tests need a B200 and call the engine through its C-ABI;
everything else runs on the CPU (oracle vs the golden fixtures, host logic,
library symbol checks).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "n-body-code_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device (B200)")
