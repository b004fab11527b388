"""Test configuration: the `gpu` marker, and builds of the oracle (the CPU
checker) and of the product library when they are missing."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    if not os.path.exists(os.path.join(ROOT, "oracle", "lib", "liboracle.so")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "lib/liboracle.so"], check=True)
    if not os.path.exists(os.path.join(ROOT, "streamgc_b200", "lib", "libstreamgc_b200.so")):
        subprocess.run(["make", "-s", "-j4", "-C", os.path.join(ROOT, "streamgc_b200", "csrc")], check=True)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU here")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
