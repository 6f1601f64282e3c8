"""Test configuration: the `gpu` marker and import paths.

`pytest -m "not gpu"` runs everything that needs no CUDA device (the oracle, host logic, the C ABI's exports);
`pytest -m gpu` runs the parity tests of the sm_100a kernels against the CPU oracle on a B200.
"""

import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "livox-warp_b200", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (sm_100a); calls the C ABI of liblivoxb200.so")
