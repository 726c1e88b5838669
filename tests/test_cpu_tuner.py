"""The lane kernel's online autotuner (kache-hash_b200/csrc/seg_tuner.hpp): compiled with g++ and run on the CPU
against a synthetic cost per launch shape (tests/tuner_check.cpp): its search order over segment lengths and block
counts, the candidate it settles on, its periodic retries, and that it follows a cost that changes."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_tuner_search_and_settling(tmp_path):
    exe = str(tmp_path / "tuner_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "kache-hash_b200", "csrc"),
                    os.path.join(ROOT, "tests", "tuner_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
