"""Shared test setup: markers and import paths.

Tests marked ``gpu`` need a CUDA device and the built library; everything
else runs on the CPU (the oracle, host logic, ABI symbol checks).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "watersim-v1_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libwatersim.so")
    config.addinivalue_line("markers", "slow: long-running CPU test")
