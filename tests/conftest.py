"""Shared test setup: import paths for the package, the built module and the oracle, and
the ``gpu`` marker (tests that need a CUDA device; run with ``-m gpu``)."""

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "mdelast_b200", "lib")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
