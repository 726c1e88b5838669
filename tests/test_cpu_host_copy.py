"""The host's streaming-store gather (kache-hash_b200/csrc/host_copy.hpp), which fills the page-locked staging
buffers that the copy engine reads: compiled with g++ and run on the CPU against a plain memcpy gather
(tests/host_copy_check.cpp)."""
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_stream_writer_gathers_as_memcpy(tmp_path):
    exe = str(tmp_path / "host_copy_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I" + os.path.join(ROOT, "kache-hash_b200", "csrc"),
                    os.path.join(ROOT, "tests", "host_copy_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
