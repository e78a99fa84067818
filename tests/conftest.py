"""pytest configuration: the ``gpu`` marker and import paths.

Tests marked ``gpu`` need a B200 (or any sm_100a device) and the built CUDA library; the
rest run on CPU only.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "master-rad_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a) and the built library")
    config.addinivalue_line("markers", "slow: full-size (million-primitive) cases")
