"""Test configuration: the `gpu` marker and import paths.

Tests marked `gpu` need an sm_100 device and the built CUDA library; everything else runs on CPU.
"""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

# Where the reference's own fixtures are read in place, when this machine has them.
REFERENCE = os.environ.get("QM_REFERENCE_ROOT", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built CUDA library")


def reference_file(relative):
    path = os.path.join(REFERENCE, relative)
    if not os.path.exists(path):
        pytest.skip(f"reference file {relative} not present on this machine")
    return path
