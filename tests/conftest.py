"""Shared test setup: the `gpu` marker and import paths.

Tests marked `gpu` need a CUDA device and run the product library
(lbgpu-prime-dev_b200/lib/liblbx.so) against the CPU oracle in oracle/.
Everything else runs on a CPU-only machine.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "lbgpu-prime-dev_b200")
for p in (os.path.join(ROOT, "oracle"), PKG, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
