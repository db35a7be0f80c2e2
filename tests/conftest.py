"""Test configuration: registers the ``gpu`` marker.

``-m "not gpu"`` runs the oracle pins, the host logic (plan execution in
numpy, C-ABI exports, argument validation) and needs no GPU; ``-m gpu``
runs the parity tests through the C ABI on a B200.
"""

from __future__ import annotations

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built extension")
