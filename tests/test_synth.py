"""The seeded FASTQ generator: exact size, determinism, thread-count invariance."""
import dataclasses

import numpy as np

from empanada_b200 import synth


def test_size_formula_and_format():
    w = dataclasses.replace(synth.SMALL, n_reads=1234, genome_len=10_000, read_len=33)
    data = synth.fastq_bytes(w)
    assert len(data) == synth.fastq_size(w)
    lines = data.split(b"\n")
    assert lines[-1] == b""
    assert len(lines) == 4 * 1234 + 1
    assert lines[0] == b"@r0" and lines[4 * 1233] == b"@r1233"
    assert all(len(lines[4 * i + 1]) == 33 and set(lines[4 * i + 1]) <= set(b"ACGT") for i in range(1234))
    assert all(lines[4 * i + 2] == b"+" and lines[4 * i + 3] == b"I" * 33 for i in range(1234))


def test_deterministic_across_threads():
    w = dataclasses.replace(synth.SMALL, n_reads=200_000, genome_len=100_000, read_len=50, sub_rate=0.01)
    a = np.empty(synth.fastq_size(w), dtype=np.uint8)
    b = np.empty_like(a)
    synth.fastq_into(w, a, threads=1)
    synth.fastq_into(w, b, threads=4)
    assert (a == b).all()
    c = synth.fastq_bytes(dataclasses.replace(w, seed=w.seed + 1))
    assert c != a.tobytes()


def test_repeat_families_are_planted():
    w = dataclasses.replace(synth.OUT_OF_CORE, genome_len=200_000, n_reads=10)
    g = synth.genome(w)
    assert len(g) == 200_000 and set(g) <= set(b"ACGT")
    g0 = synth.genome(dataclasses.replace(w, repeat_frac=0.0))
    diff = sum(1 for x, y in zip(g, g0) if x != y)
    assert diff > 0.02 * len(g)  # ~5 % of the genome overwritten by repeat copies
