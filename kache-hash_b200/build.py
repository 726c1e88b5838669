"""Builds libkache_b200.so in-tree (under _build/) for sm_100a with nvcc, one object per translation unit, in
parallel, then links them. Objects are rebuilt only when a source or header is newer.

    python kache-hash_b200/build.py [--force]
"""
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "libkache_b200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++20", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0)


def build(force=False, verbose=False):
    os.makedirs(OUT, exist_ok=True)
    units = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    h_time = _newest(headers + [__file__])

    def compile_one(src):
        obj = os.path.join(OUT, os.path.basename(src) + ".o")
        if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), h_time):
            return obj
        cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [NVCC] + FLAGS + ["-x", "cu"] + ARCH + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, file=sys.stderr)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, len(units))) as ex:
        objs = list(ex.map(compile_one, units))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread", "-Xlinker", "-Bsymbolic"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stderr}")
    build_facade_check(headers, force)
    build_counter_check(force)
    return LIB


def build_facade_check(headers, force=False):
    """The C++ template surface's check program (tests/facade_check.cu), linked against the library."""
    src = os.path.join(ROOT, "tests", "facade_check.cu")
    exe = os.path.join(OUT, "facade_check")
    if not os.path.exists(src):
        return None
    if not force and os.path.exists(exe) and os.path.getmtime(exe) >= max(_newest(headers), os.path.getmtime(src), os.path.getmtime(LIB)):
        return exe
    cmd = [NVCC] + ARCH + FLAGS + [src, "-o", exe, "-L" + OUT, "-lkache_b200", "-Xlinker", "-rpath=" + OUT]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stderr}")
    return exe


def build_counter_check(force=False):
    """The counter's C++ surface's check program (tests/counter_check.cpp): plain C++ over include/Kmer_Set_Counter.hpp,
    linked against the library as a C++ caller of the reference's counter would be."""
    src = os.path.join(ROOT, "tests", "counter_check.cpp")
    exe = os.path.join(OUT, "counter_check")
    hdr = os.path.join(ROOT, "include", "Kmer_Set_Counter.hpp")
    if not os.path.exists(src):
        return None
    if not force and os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(src), os.path.getmtime(hdr), os.path.getmtime(LIB)):
        return exe
    cmd = [os.environ.get("CXX", "g++"), "-std=c++20", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"), src, "-o", exe,
           "-L" + OUT, "-lkache_b200", "-Wl,-rpath=" + OUT, "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"g++ failed on {src}:\n{r.stderr}")
    return exe


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
