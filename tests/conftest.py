"""Pytest configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on a CPU-only host (oracle pins, host logic, the C-ABI
export check); `-m gpu` runs the CUDA parity tests on a B200.
"""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "splat.js_b200"), os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built CUDA library")
