"""Shared pytest configuration.

Tests marked ``gpu`` need a CUDA device and the built ``libmetalmom.so``;
everything else runs on the CPU.
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built CUDA library")
    config.addinivalue_line("markers", "slow: longer-running CPU test")
