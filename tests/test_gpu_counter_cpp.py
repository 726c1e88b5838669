"""The counter's C++ surface (include/Kmer_Set_Counter.hpp, the reference's class and signatures) through its check
program tests/counter_check.cpp, built with the library: files and a pipe, priming twice, count_of in both
orientations and cases, histograms, sizes, the constructor's invalid arguments."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "kache-hash_b200", "_build", "counter_check")


def test_counter_cpp_surface(tmp_path):
    assert os.path.exists(EXE), "build the library first (it builds the check program)"
    r = subprocess.run([EXE, str(tmp_path)], capture_output=True, text=True, timeout=600)
    print(r.stdout, r.stderr)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout + r.stderr
