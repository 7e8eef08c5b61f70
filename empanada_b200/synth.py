"""Seeded synthetic FASTQ workloads for the read-overlap path.

The generator itself is C (``csrc/synth_reads.c``, built into
``libempanada_synth.so``); this module binds it with ctypes and names the
workloads the overlap path is measured on:

``small``       1 Mbp uniform genome, 100,000 error-free 150 bp reads, -o 31,
                default block sizes.
``larger``      5 Mbp genome, 1.2M 250 bp reads with 0.1 % substitutions,
                -o 75 -m 8g -r 12g -b 16m -c 64m.
``out_of_core`` 100 Mbp genome with 5 % repeat families (1-5 kbp copies,
                1 % divergence, 2-50 copies), 150 bp reads at 50x;
                -m 1g -r 1g (block streaming) or HBM-sized blocks.

Every read is reverse-complemented with probability 0.5 and gets constant
quality 'I'.
"""
from __future__ import annotations

import ctypes
import dataclasses
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libempanada_synth.so")


class _Params(ctypes.Structure):
    _fields_ = [
        ("seed", ctypes.c_uint64),
        ("genome_len", ctypes.c_uint64),
        ("n_reads", ctypes.c_uint64),
        ("read_len", ctypes.c_int32),
        ("n_threads", ctypes.c_int32),
        ("sub_rate", ctypes.c_double),
        ("rc_prob", ctypes.c_double),
        ("repeat_frac", ctypes.c_double),
        ("rep_min_len", ctypes.c_int32),
        ("rep_max_len", ctypes.c_int32),
        ("rep_min_copies", ctypes.c_int32),
        ("rep_max_copies", ctypes.c_int32),
        ("rep_divergence", ctypes.c_double),
    ]


@dataclasses.dataclass(frozen=True)
class Workload:
    name: str
    seed: int
    genome_len: int
    n_reads: int
    read_len: int
    sub_rate: float = 0.0
    rc_prob: float = 0.5
    repeat_frac: float = 0.0
    rep_min_len: int = 1000
    rep_max_len: int = 5000
    rep_min_copies: int = 2
    rep_max_copies: int = 50
    rep_divergence: float = 0.01
    # the reference CLI options the workload is run with
    min_ovlp: int = 31
    map_mem: str = "1g"
    reduce_mem: str = "1g"
    base_blocksz: str = "32m"
    kv_chunksz: str = "64m"

    def cli_args(self) -> list[str]:
        return ["-o", str(self.min_ovlp), "-m", self.map_mem, "-r", self.reduce_mem,
                "-b", self.base_blocksz, "-c", self.kv_chunksz]

    def scaled(self, n_reads: int, name: str | None = None) -> "Workload":
        """Same genome and error model with fewer reads (a bounded sample)."""
        return dataclasses.replace(self, n_reads=n_reads, name=name or f"{self.name}[:{n_reads}]")

    def sampled(self, n_reads: int) -> "Workload":
        """A bounded sample at the same coverage: n_reads reads from a genome
        shrunk by the same factor (same read length, error and repeat model,
        options and seed), so each read meets as many overlaps as in the full
        workload."""
        if n_reads >= self.n_reads:
            return self
        g = max(4 * self.read_len, round(self.genome_len * n_reads / self.n_reads))
        return dataclasses.replace(self, n_reads=n_reads, genome_len=g,
                                   name=f"{self.name} [sample: {n_reads} reads of a {g} bp genome, same coverage]")


SMALL = Workload("small: 1 Mbp genome, 100k x 150 bp error-free reads, -o 31", seed=1,
                 genome_len=1_000_000, n_reads=100_000, read_len=150, min_ovlp=31)
LARGER = Workload("larger: 5 Mbp genome, 1.2M x 250 bp reads, 0.1% subs, -o 75 -m 8g -r 12g -b 16m -c 64m",
                  seed=2, genome_len=5_000_000, n_reads=1_200_000, read_len=250, sub_rate=0.001,
                  min_ovlp=75, map_mem="8g", reduce_mem="12g", base_blocksz="16m", kv_chunksz="64m")
OUT_OF_CORE = Workload("out_of_core: 100 Mbp genome (5% repeat families), 150 bp reads at 50x, -m 1g -r 1g",
                       seed=3, genome_len=100_000_000, n_reads=33_333_333, read_len=150,
                       repeat_frac=0.05, min_ovlp=31, map_mem="1g", reduce_mem="1g")
OUT_OF_CORE_HBM = dataclasses.replace(OUT_OF_CORE, name="out_of_core, HBM-sized blocks: as out_of_core with "
                                      "-m 160g -r 160g", map_mem="160g", reduce_mem="160g")
WORKLOADS = {"small": SMALL, "larger": LARGER, "out_of_core": OUT_OF_CORE, "out_of_core_hbm": OUT_OF_CORE_HBM}


def batched_sets(n_sets: int = 256, seed: int = 4, genome_min: int = 50_000, genome_max: int = 5_000_000,
                 len_min: int = 100, len_max: int = 300, cov_min: float = 10.0, cov_max: float = 80.0,
                 sub_rate: float = 0.001, min_ovlp: int = 31) -> list[Workload]:
    """Independent read sets of a batch: genome size log-uniform in
    [genome_min, genome_max], read length uniform in [len_min, len_max]
    (fixed within a set), coverage uniform in [cov_min, cov_max], uniform
    substitutions at sub_rate, each set with its own seed."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_sets):
        g = int(round(np.exp(rng.uniform(np.log(genome_min), np.log(genome_max)))))
        L = int(rng.integers(len_min, len_max + 1))
        cov = float(rng.uniform(cov_min, cov_max))
        n = max(1, int(g * cov / L))
        out.append(Workload(f"set{k}: {g} bp genome, {n} x {L} bp", seed=seed * 1_000_003 + k, genome_len=g,
                            n_reads=n, read_len=L, sub_rate=sub_rate, min_ovlp=min_ovlp))
    return out

_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise RuntimeError(f"{_LIB_PATH} is missing; run __graft_entry__.build() first")
        lib = ctypes.CDLL(_LIB_PATH)
        lib.emp_synth_fastq_size.restype = ctypes.c_uint64
        lib.emp_synth_fastq_size.argtypes = [ctypes.c_uint64, ctypes.c_int32]
        lib.emp_synth_fastq.restype = ctypes.c_uint64
        lib.emp_synth_fastq.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p, ctypes.c_uint64]
        lib.emp_synth_genome.restype = ctypes.c_int
        lib.emp_synth_genome.argtypes = [ctypes.POINTER(_Params), ctypes.c_void_p]
        _lib = lib
    return _lib


def _params(w: Workload, threads: int = 0) -> _Params:
    return _Params(w.seed, w.genome_len, w.n_reads, w.read_len, threads, w.sub_rate, w.rc_prob,
                   w.repeat_frac, w.rep_min_len, w.rep_max_len, w.rep_min_copies, w.rep_max_copies,
                   w.rep_divergence)


def fastq_size(w: Workload) -> int:
    return int(_load().emp_synth_fastq_size(w.n_reads, w.read_len))


def fastq_into(w: Workload, out: np.ndarray, threads: int = 0) -> int:
    """Write the workload's FASTQ into a uint8 array (e.g. pinned host memory)."""
    need = fastq_size(w)
    if out.dtype != np.uint8 or out.size < need or not out.flags.c_contiguous:
        raise ValueError("output must be a contiguous uint8 array of at least fastq_size() bytes")
    p = _params(w, threads)
    got = _load().emp_synth_fastq(ctypes.byref(p), out.ctypes.data, out.size)
    if got != need:
        raise RuntimeError("synthetic FASTQ generation failed")
    return need


def fastq_bytes(w: Workload, threads: int = 0) -> bytes:
    buf = np.empty(fastq_size(w), dtype=np.uint8)
    fastq_into(w, buf, threads)
    return buf.tobytes()


def write_fastq(w: Workload, path: str, threads: int = 0) -> int:
    buf = np.empty(fastq_size(w), dtype=np.uint8)
    fastq_into(w, buf, threads)
    buf.tofile(path)
    return buf.size


def genome(w: Workload) -> bytes:
    g = np.empty(w.genome_len, dtype=np.uint8)
    p = _params(w)
    if _load().emp_synth_genome(ctypes.byref(p), g.ctypes.data) != 0:
        raise RuntimeError("genome generation failed")
    return g.tobytes()
