"""The FASTA/FASTQ reader of the counter (kache_b200_fastx_read), without a GPU: its sequences equal a plain
sequential parse over FASTA and FASTQ, multi-line records, CRLF line ends, a missing last line end, pipes and batch
sizes from one base up; malformed and gzip input are refused (reference test/counter.cpp:245-311)."""
import ctypes
import os
import threading

import numpy as np
import pytest

import kache

SEQS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_char_p), ctypes.POINTER(ctypes.c_size_t), ctypes.c_size_t)


def read(path, batch=1 << 20):
    f = kache.lib().kache_b200_fastx_read
    f.restype, f.argtypes = ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, SEQS_FN, ctypes.c_void_p]
    out, sizes = [], []

    def cb(ctx, seqs, lens, n):
        sizes.append(n)
        for i in range(n):
            out.append(ctypes.string_at(ctypes.cast(seqs, ctypes.POINTER(ctypes.c_void_p))[i], lens[i]))
        return 0

    rc = f(path.encode(), batch, SEQS_FN(cb), None)
    return rc, out, sizes


def records(seed, n=50):
    rng = np.random.default_rng(seed)
    return [bytes(rng.choice(list(b"ACGTNacgt"), size=int(rng.integers(1, 900))).astype(np.uint8)) for _ in range(n)]


def fasta(seqs, width, eol=b"\n", last_eol=True):
    out = b""
    for i, s in enumerate(seqs):
        out += b">seq" + str(i).encode() + b" desc" + eol
        for j in range(0, len(s), width):
            out += s[j:j + width] + eol
    return out if last_eol else out.rstrip(b"\r\n")


def fastq(seqs, eol=b"\n", last_eol=True):
    out = b""
    for i, s in enumerate(seqs):
        out += b"@r" + str(i).encode() + eol + s + eol + b"+" + eol + b"I" * len(s) + eol
    return out if last_eol else out.rstrip(b"\r\n")


@pytest.mark.parametrize("width", [1, 60, 10_000])
@pytest.mark.parametrize("eol", [b"\n", b"\r\n"])
@pytest.mark.parametrize("last_eol", [True, False])
def test_fasta(tmp_path, width, eol, last_eol):
    seqs = records(1)
    p = tmp_path / "x.fa"
    p.write_bytes(fasta(seqs, width, eol, last_eol))
    for batch in (1, 1000, 1 << 24):
        rc, got, sizes = read(str(p), batch)
        assert rc == kache.KACHE_OK and got == seqs


@pytest.mark.parametrize("eol", [b"\n", b"\r\n"])
@pytest.mark.parametrize("last_eol", [True, False])
def test_fastq(tmp_path, eol, last_eol):
    seqs = records(2)
    p = tmp_path / "x.fq"
    p.write_bytes(fastq(seqs, eol, last_eol))
    rc, got, _ = read(str(p), 777)
    assert rc == kache.KACHE_OK and got == seqs


def test_empty_records_skipped_and_empty_file(tmp_path):
    p = tmp_path / "e.fa"
    p.write_bytes(b">a\n>b\nACGT\n>c\n\n>d\nTT\nGG\n")
    assert read(str(p))[1] == [b"ACGT", b"TTGG"]
    q = tmp_path / "empty.fa"
    q.write_bytes(b"")
    assert read(str(q))[:2] == (kache.KACHE_OK, [])


def test_pipe(tmp_path):
    seqs = records(3, 400)
    data = fasta(seqs, 70)
    fifo = str(tmp_path / "pipe")
    os.mkfifo(fifo)

    def writer():
        with open(fifo, "wb") as w:
            for i in range(0, len(data), 4096):
                w.write(data[i:i + 4096])

    t = threading.Thread(target=writer)
    t.start()
    rc, got, _ = read(fifo, 5000)
    t.join()
    assert rc == kache.KACHE_OK and got == seqs


@pytest.mark.parametrize("content", [b"ACGT\n", b"@r\nACGT\n-\nIIII\n", b"@r\nACGT\n+\nIII\n", b"@r\nACGT\n", b"\x1f\x8b\x08\x00", b">a\nAC\n@b\n"[0:0] + b"x>a\n"])
def test_malformed(tmp_path, content):
    p = tmp_path / "bad"
    p.write_bytes(content)
    assert read(str(p))[0] == kache.KACHE_EINVAL


def test_unreadable():
    assert read("/nonexistent/file.fa")[0] == kache.KACHE_EINVAL
