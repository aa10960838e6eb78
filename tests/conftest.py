"""Test configuration: the package directory and the oracle on sys.path, the ``gpu`` marker."""

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
for sub in ("gpu-quantum-interferometry-solver_b200", "oracle"):
    path = str(ROOT / sub)
    if path not in sys.path:
        sys.path.insert(0, path)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
