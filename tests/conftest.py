"""Test configuration: the `gpu` marker and import paths.

`-m "not gpu"` runs on any host: the oracle against the reference's
known-answer tests, host-side logic, and the C-ABI library's exports.
`-m gpu` runs the CUDA parity tests (needs a CUDA device).
"""

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running CPU test")
