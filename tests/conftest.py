"""Test configuration: the `gpu` marker (tests that need a B200), and the import paths of the package's Python
binding (kache-hash_b200/), of the checker (oracle/) and of the synthetic workloads (tests/synth.py)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "kache-hash_b200"), os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (a B200); runs the CUDA path through the C interface")
