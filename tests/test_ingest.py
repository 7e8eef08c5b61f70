"""FASTQ input from files without a GPU (emp_fastq_load, the reader behind
emp_job_feed_files, emp_run_files and the CLI): plain, gzip (one or more
members) and BGZF files, several files in order with a newline added where a
file ends inside a line, missing files, and damaged compressed input."""
import gzip
import os
import struct
import zlib

import numpy as np
import pytest

import empanada_b200
from empanada_b200 import EmpError

BGZF_EOF = bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")


def bgzf(data: bytes, block: int = 65280, eof: bool = True, level: int = 6) -> bytes:
    """BGZF (the SAM/BAM blocked gzip): gzip members of at most 64 KiB, each
    with the 'BC' extra subfield giving its size."""
    out = bytearray()
    for o in range(0, len(data), block):
        piece = data[o:o + block]
        c = zlib.compressobj(level, zlib.DEFLATED, -15)
        body = c.compress(piece) + c.flush()
        bsize = 18 + len(body) + 8
        out += bytes([0x1F, 0x8B, 8, 4, 0, 0, 0, 0, 0, 0xFF]) + struct.pack("<HBBHH", 6, 66, 67, 2, bsize - 1)
        out += body + struct.pack("<II", zlib.crc32(piece) & 0xFFFFFFFF, len(piece))
    if eof:
        out += BGZF_EOF
    return bytes(out)


def fastq(n: int, L: int = 100, seed: int = 1, trailing_newline: bool = True) -> bytes:
    rng = np.random.default_rng(seed)
    bases = np.frombuffer(b"ACGT", dtype=np.uint8)[rng.integers(0, 4, size=(n, L))]
    recs = [b"@r%d\n%s\n+\n%s\n" % (i, bases[i].tobytes(), b"I" * L) for i in range(n)]
    s = b"".join(recs)
    return s if trailing_newline else s[:-1]


def write(path, data: bytes):
    path.write_bytes(data)
    return str(path)


def test_plain_gzip_and_bgzf_read_the_same_bytes(tmp_path):
    data = fastq(3000)
    plain = write(tmp_path / "a.fq", data)
    gz = write(tmp_path / "a.fq.gz", gzip.compress(data))
    bg = write(tmp_path / "a.fq.bgz", bgzf(data))
    for p in (plain, gz, bg):
        assert empanada_b200.load_fastq(p) == data, p


def test_multi_member_gzip_is_one_stream(tmp_path):
    a, b = fastq(500, seed=2), fastq(700, seed=3)
    p = write(tmp_path / "m.fq.gz", gzip.compress(a) + gzip.compress(b))
    assert empanada_b200.load_fastq(p) == a + b


def test_large_inputs_span_many_pieces(tmp_path):
    """More than one reader piece: a gzip stream (size unknown, the buffer
    grows) and a BGZF file inflated by several host threads."""
    data = fastq(120_000, L=150, seed=4)  # about 38 MB
    gz = write(tmp_path / "big.fq.gz", gzip.compress(data, compresslevel=1))
    bg = write(tmp_path / "big.fq.bgz", bgzf(data))
    assert empanada_b200.load_fastq(gz) == data
    assert empanada_b200.load_fastq(bg) == data


def test_large_plain_files_read_in_slices(tmp_path):
    """Plain files above the 16 MiB slice size are read by several threads at
    once; the pieces land in order, across files too."""
    a = fastq(300_000, L=150, seed=9)  # about 95 MB: several slices
    b = fastq(70_001, L=101, seed=10, trailing_newline=False)  # not a multiple of the page size
    pa, pb = write(tmp_path / "a.fq", a), write(tmp_path / "b.fq", b)
    assert empanada_b200.load_fastq(pa) == a
    assert empanada_b200.load_fastq([pb, pa, pb]) == b + b"\n" + a + b


def test_files_in_order_with_newlines_between(tmp_path):
    a = fastq(10, seed=5, trailing_newline=False)
    b = fastq(20, seed=6)
    c = fastq(5, seed=7, trailing_newline=False)
    pa = write(tmp_path / "a.fq", a)
    pb = write(tmp_path / "b.fq.gz", gzip.compress(b))
    pc = write(tmp_path / "c.fq.bgz", bgzf(c))
    empty = write(tmp_path / "e.fq", b"")
    missing = str(tmp_path / "absent.fq")
    # a newline goes after a file that ends inside a line when bytes follow;
    # the last file keeps its missing newline; empty and missing files add nothing
    assert empanada_b200.load_fastq([pa, empty, missing, pb, pc]) == a + b"\n" + b + c
    assert empanada_b200.load_fastq([pb, pa]) == b + a
    assert empanada_b200.load_fastq([pa, empty]) == a
    assert empanada_b200.load_fastq([missing]) == b""
    assert empanada_b200.load_fastq([]) == b""


def test_damaged_or_unreadable_input_is_an_error(tmp_path):
    data = fastq(2000, seed=8)
    z = gzip.compress(data)
    trunc = write(tmp_path / "t.fq.gz", z[: len(z) // 2])
    with pytest.raises(EmpError) as e:
        empanada_b200.load_fastq(trunc)
    assert e.value.code == -5  # EMP_E_FORMAT
    b = bytearray(bgzf(data))
    b[40] ^= 0xFF  # inside the first block's deflate data
    bad = write(tmp_path / "bad.fq.bgz", bytes(b))
    with pytest.raises(EmpError) as e:
        empanada_b200.load_fastq(bad)
    assert e.value.code == -5
    (tmp_path / "dir.fq").mkdir()
    with pytest.raises(EmpError) as e:
        empanada_b200.load_fastq(str(tmp_path / "dir.fq"))
    assert e.value.code == -7  # EMP_E_IO


def test_bgzf_blocks_across_reads_of_the_file(tmp_path):
    """Compressed bytes are read 16 MiB at a time and blocks parsed in memory:
    blocks that straddle those reads, a file cut inside a block, and bytes
    after the last block that are not a block."""
    data = fastq(120_000, L=150, seed=12)  # about 38 MB
    z = bgzf(data, level=0)  # stored blocks: as large as the data, so several reads
    p = write(tmp_path / "s.fq.bgz", z)
    assert empanada_b200.load_fastq(p) == data
    for bad in (z[: len(z) - 28 - 1000], z + b"not a block"):
        with pytest.raises(EmpError) as e:
            empanada_b200.load_fastq(write(tmp_path / "bad.fq.bgz", bad))
        assert e.value.code == -5  # EMP_E_FORMAT


def test_bgzf_without_eof_block_and_gzip_with_trailing_garbage(tmp_path):
    data = fastq(400, seed=9)
    p = write(tmp_path / "noeof.fq.bgz", bgzf(data, eof=False))
    assert empanada_b200.load_fastq(p) == data
    g = write(tmp_path / "junk.fq.gz", gzip.compress(data) + b"not gzip")
    with pytest.raises(EmpError):
        empanada_b200.load_fastq(g)


def test_host_copies_beyond_2_gib():
    """load_fastq hands out inputs above 2 GiB (a copy whose size is a C int
    fails there)."""
    import psutil

    n = (1 << 31) + 64
    if psutil.virtual_memory().available < 3 * n:
        pytest.skip("not enough free host memory for a 2 GiB copy")
    a = np.zeros(n, dtype=np.uint8)
    a[[0, (1 << 31) - 1, 1 << 31, n - 1]] = [65, 67, 71, 84]
    b = empanada_b200.host_bytes(a.ctypes.data, n)
    assert len(b) == n and b[0] == 65 and b[(1 << 31) - 1] == 67 and b[1 << 31] == 71 and b[-1] == 84
    assert empanada_b200.host_bytes(a.ctypes.data, 0) == b""
