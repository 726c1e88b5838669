"""The C++ template surface (Streaming_Kmer_Hash_Table.cuh) through its check program tests/facade_check.cu, built
with the library: user device functors, host lookup and iteration callbacks, single finds, resizing."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "kache-hash_b200", "_build", "facade_check")


def test_facade_check():
    assert os.path.exists(EXE), "build the library first (it builds the check program)"
    r = subprocess.run([EXE], capture_output=True, text=True, timeout=300)
    print(r.stdout, r.stderr)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
