"""Test configuration: import paths and the `gpu` marker.

`-m "not gpu"` runs on a machine without a GPU: the oracle against the golden
vectors and the reference, the C ABI's host-side behaviour, and index files.
`-m gpu` runs the parity tests proper, through the C ABI, on a CUDA device.
"""

import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "neural-sparse-cpp_b200", "python"), os.path.join(ROOT, "oracle"),
          os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
